"""The oracle pinned against the reference's golden logs and analytic known answers (CPU)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from matjes_b200.deck import Deck, square_areal, square_film, triangular

GOLD = os.path.join(os.path.dirname(__file__), "golden", "isolated_spin_precession.json")


def _precession_deck():
    g = json.load(open(GOLD))["deck"]
    return Deck(L=tuple(g["L"]), periodic=(1, 1, 0), areal=square_areal(), atoms=[((0, 0, 0), 1, g["mu_s"])],
                J=[(1, 1, 1, g["J1"])], B_ext=tuple(g["B_ext"]))


def _hbar_of_log(rows):
    """The log predates the current hbar constant: recover it from step 1 only."""
    my = rows[0, 4]
    theta = my / np.sqrt(1.0 - my * my)
    return O.MUB * 10.0 * 1.0 / theta


def test_euler_matches_reference_golden_log():
    """tests/serial/isolated_spin_precession/Euler/REF: 50 Euler steps, every row."""
    rows = np.array(json.load(open(GOLD))["euler"]["rows"])
    hb = _hbar_of_log(rows)
    assert abs(hb - O.HBAR) < 1e-4  # same constant up to the older CODATA value
    M = O.Model(_precession_deck())
    m = np.tile([1.0, 0.0, 0.0], (16, 1))
    for k in range(50):
        E = M.run(m, 1, integrator="euler", timestep=1.0 * O.HBAR / hb, alpha=0.0, energies=True)
        avg = m.mean(0)
        # the log prints 12 significant digits
        assert abs(avg[0] - rows[k, 3]) < 2e-12
        assert abs(avg[1] - rows[k, 4]) < 2e-12
        assert abs(avg[2] - rows[k, 5]) < 1e-20
        assert abs(E[0] / 16 - rows[k, 1]) < 1e-18  # E_av = -z J per site, Zeeman 0 for m in-plane


def test_heun_reproduces_reference_log_qualitatively():
    """Heun/EM.dat comes from an older Heun that also drifted Mz by 5e-9/step;
    the current scheme (stage dt = timestep/2, corrector from the predictor)
    reproduces its precession to 3e-8 with a doubled timestep."""
    g = json.load(open(GOLD))
    erows = np.array(g["euler"]["rows"])
    hrows = np.array(g["heun"]["rows"])
    hb = _hbar_of_log(erows)
    M = O.Model(_precession_deck())
    m = np.tile([1.0, 0.0, 0.0], (16, 1))
    for k in range(50):
        M.run(m, 1, integrator="heun", timestep=2.0 * O.HBAR / hb, alpha=0.0)
        avg = m.mean(0)
        assert abs(avg[1] - hrows[k, 4]) < 3e-8 * (k + 1)
        assert abs(avg[0] - hrows[k, 3]) < 3e-9 * (k + 1)
    # one Heun step advances about two Euler steps (F2 of the reference)
    assert abs(hrows[0, 4] - erows[1, 4]) < 1e-12


def test_ferromagnet_energies_per_shell():
    deck = triangular((12, 12), J=(1e-3, -0.1e-3, -0.05e-3), Dv=0.2e-3, Kv=-0.05e-3, Bz=1.0)
    M = O.Model(deck)
    m = np.tile([0.0, 0.0, 1.0], (deck.nsites, 1))
    B, e = M.field(m)
    # directed pairs, left-assigned: E_i = -sum_shells z_s J_s + K + Zeeman (DMI vanishes)
    e_exp = -(6 * 1e-3 + 6 * -0.1e-3 + 6 * -0.05e-3) + (-0.05e-3) - O.MUB * 2.0 * 1.0
    assert np.allclose(e, e_exp, rtol=1e-14, atol=0)
    assert abs(M.energy(m) - deck.nsites * e_exp) < 1e-12 * abs(deck.nsites * e_exp)
    # field: 2 sum_s z_s J_s + 2|K| + mu_B mu_s B along z
    bz = 2 * (6 * 1e-3 + 6 * -0.1e-3 + 6 * -0.05e-3) + 2 * 0.05e-3 + O.MUB * 2.0
    assert np.allclose(B[:, 2], bz, rtol=1e-14) and np.abs(B[:, :2]).max() < 1e-18


@pytest.mark.parametrize("q", [0.1, -0.25, 0.6])
def test_cycloid_energy_and_dmi_handedness(q):
    L = 32
    deck = square_film((L, L, 1), Jv=1e-3, Dv=0.3e-3, Kv=0.0, Bz=0.0)
    M = O.Model(deck)
    x = np.arange(L)
    qq = 2 * np.pi * round(q * L / (2 * np.pi)) / L  # commensurate with the periodic box
    ang = np.tile(qq * x, L)
    m = np.stack([np.sin(ang), np.zeros_like(ang), np.cos(ang)], 1)
    e = M.field(m)[1]
    # exchange -J(2 cos q + 2), DMI with d = z x r: c_H_D D (2 sin q) = -2 D sin q
    e_exp = -1e-3 * (2 * np.cos(qq) + 2) - 2 * 0.3e-3 * np.sin(qq)
    assert np.allclose(e, e_exp, rtol=1e-12, atol=1e-18)


def test_sib_precession_is_a_cayley_rotation():
    """SIB on a single precessing spin rotates by 2 atan(theta/2) per step and keeps |m|."""
    deck = Deck(L=(1, 1, 1), periodic=(0, 0, 0), areal=square_areal(), atoms=[((0, 0, 0), 1, 2.0)], B_ext=(0, 0, 5.0))
    M = O.Model(deck)
    m = np.array([[1.0, 0.0, 0.0]])
    dt = 0.7
    M.run(m, 10, integrator="sib", timestep=dt, alpha=0.0)
    theta = O.MUB * 2.0 * 5.0 * dt / O.HBAR
    phi = 10 * 2 * np.arctan(theta / 2)
    assert np.allclose(m[0], [np.cos(phi), np.sin(phi), 0.0], atol=1e-15)
    assert abs(np.linalg.norm(m[0]) - 1.0) < 1e-15


def test_sib_damped_relaxation_preserves_norm():
    deck = square_film((16, 16, 1))
    M = O.Model(deck)
    rng = np.random.default_rng(5)
    m = rng.normal(size=(deck.nsites, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    E = M.run(m, 200, integrator="sib", timestep=0.5, alpha=0.5, energies=True)
    assert np.abs(np.linalg.norm(m, axis=1) - 1).max() < 1e-13
    assert E[-1] < E[0]  # damped dynamics lowers the energy


def test_dipolar_fft_route_matches_explicit_sum_open_boundaries():
    """With open boundaries the FFT-route K (doubled grid) equals the explicit pair sum."""
    deck = square_film((5, 4, 3), Jv=0.0, Dv=0.0, Kv=0.0, Bz=0.0, periodic=(0, 0, 0), a=0.25, dip=True)
    M = O.Model(deck)
    assert M.nrep() == (10, 8, 6)
    rng = np.random.default_rng(1)
    m = rng.normal(size=(deck.nsites, 3))
    B = M.field(m)[0]
    Bx = M.dipolar_explicit(m)
    assert np.abs(B - Bx).max() < 1e-13 * np.abs(Bx).max()


def test_dipolar_periodic_grid_rule():
    """Periodic axes keep N_rep = L (images summed), open axes double (F7)."""
    deck = square_film((8, 8, 4), periodic=(1, 1, 0), a=0.25, med_z=-0.3, dip=True)
    assert O.Model(deck).nrep() == (8, 8, 8)


@pytest.mark.parametrize("dip,nrep", [(1, (8, 8, 8)), (2, (16, 16, 8))])
def test_dipolar_fft_route_equals_direct_circular_sum(dip, nrep):
    """The oracle's own FFT of the N_rep grid and the direct circular sum over it
    give the same dipolar field (reference grid rule and the zero-padded grid)."""
    deck = square_film((8, 8, 4), Jv=0.0, Dv=0.0, Kv=0.0, Bz=0.0, periodic=(1, 1, 0), a=0.25, dip=dip)
    M = O.Model(deck)
    assert M.nrep() == nrep
    m = np.random.default_rng(2).normal(size=(deck.nsites, 3))
    B_fft = M.field(m)[0]
    M.dip_direct(True)
    B_dir = M.field(m)[0]
    assert np.abs(B_fft - B_dir).max() < 1e-13 * np.abs(B_dir).max()
    assert M.energy(m) != 0.0


def test_zero_padded_grid_equals_the_explicit_pair_sum():
    """dip = 2 (every axis zero-padded to 2 L, 256 x 256 x 32 for the
    128 x 128 x 16 film): a linear convolution whose kernel sums the periodic
    images over -cut..cut for every pair, which is the explicit route
    (Energy/dipolar_magnetic.f90:181-273).  The reference's grid (periodic axes
    kept at L, images folded in circularly) sums a window shifted by one period
    for pairs at negative offsets, so it differs from the explicit sum by far
    more than rounding."""
    kw = dict(Jv=0.0, Dv=0.0, Kv=0.0, Bz=0.0, periodic=(1, 1, 0), a=0.25)
    m = np.random.default_rng(3).normal(size=(8 * 6 * 3, 3))
    padded = O.Model(square_film((8, 6, 3), dip=2, **kw))
    assert padded.nrep() == (16, 12, 6)
    Bx = padded.dipolar_explicit(m)
    assert np.abs(padded.field(m)[0] - Bx).max() < 1e-12 * np.abs(Bx).max()
    ref_rule = O.Model(square_film((8, 6, 3), dip=1, **kw))
    assert np.abs(ref_rule.field(m)[0] - Bx).max() > 1e-6 * np.abs(Bx).max()


def test_dipolar_shape_anisotropy_sign():
    deck = square_film((8, 8, 2), Jv=0.0, Dv=0.0, Kv=0.0, Bz=0.0, periodic=(1, 1, 0), a=0.25, dip=True)
    M = O.Model(deck)
    up = np.tile([0.0, 0.0, 1.0], (deck.nsites, 1))
    inplane = np.tile([1.0, 0.0, 0.0], (deck.nsites, 1))
    assert M.energy(up) > 0 > M.energy(inplane)


def test_philox_known_answers():
    """Random123 philox4x32-10 known-answer vectors."""
    assert O.philox4x32([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert O.philox4x32([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert O.philox4x32([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_box_muller_tables_are_accurate():
    """The table-driven log and sin/cos(2 pi u) of u = (w + 1/2) 2^-32 agree with
    libm (in extended precision) on every kind of word: log within 3 ulp plus
    3e-16 absolute (the absolute part for u above 1/2, where ln u cancels against
    -ln 2), sin and cos to 3e-16 absolute."""
    rng = np.random.default_rng(0)
    w = np.concatenate([rng.integers(0, 2 ** 32, 400000, dtype=np.uint64),
                        np.arange(0, 4096, dtype=np.uint64), 2 ** 32 - 1 - np.arange(0, 4096, dtype=np.uint64),
                        (np.arange(1024, dtype=np.uint64) << 22), (np.arange(1024, dtype=np.uint64) << 22) - 1,
                        (np.arange(1024, dtype=np.uint64) << 22) + 2 ** 21]) % (2 ** 32)
    w = w.astype(np.uint32)
    lg, s, c = O.tab_eval(w)
    u = (w.astype(np.longdouble) + 0.5) / np.longdouble(2.0) ** 32
    ref = np.log(u)
    err = np.abs(lg - ref).astype(np.float64)
    assert (err <= 3 * np.spacing(np.abs(ref).astype(np.float64)) + 3e-16).all()
    ang = 2 * np.longdouble(np.pi) * u
    assert np.abs(s - np.sin(ang)).astype(np.float64).max() < 3e-16
    assert np.abs(c - np.cos(ang)).astype(np.float64).max() < 3e-16


def test_philox_normals_statistics():
    z = O.philox_normals(seed=7, step=3, stream=0, site0=0, n=200000).ravel()
    assert abs(z.mean()) < 5 * 1 / np.sqrt(z.size)
    assert abs(z.var() - 1) < 5 * np.sqrt(2 / z.size)
    kurt = ((z - z.mean()) ** 4).mean() / z.var() ** 2
    assert abs(kurt - 3) < 0.05
    other = O.philox_normals(seed=7, step=4, stream=0, site0=0, n=1000)
    assert not np.allclose(other, z[:3000].reshape(-1, 3))


def test_thermal_noise_sigma_matches_reference_formula():
    """One Euler step of a single spin at alpha>0, T>0 with injected unit noise
    adds DT dt/hbar with DT the LLG torque of b = sigma n, sigma = sqrt(alpha kT hbar/dt)."""
    deck = Deck(L=(1, 1, 1), periodic=(0, 0, 0), areal=square_areal(), atoms=[((0, 0, 0), 1, 2.0)])
    M = O.Model(deck)
    m = np.array([[1.0, 0.0, 0.0]])
    n = np.array([[[0.0], [1.0], [0.5]]])  # [nbuf][3][N]
    alpha, T, dt = 0.2, 30.0, 0.1
    M.run(m, 1, integrator="euler", timestep=dt, alpha=alpha, temperature=T, noise="inject", inject=n)
    sigma = np.sqrt(alpha * T * O.KB * O.HBAR / dt)
    b = sigma * np.array([0.0, 1.0, 0.5])
    DT = O.llg_torque(b[None], alpha, np.array([[1.0, 0.0, 0.0]]))[0]
    t = np.array([1.0, 0.0, 0.0]) + DT * dt / O.HBAR
    assert np.allclose(m[0], t / np.linalg.norm(t), atol=1e-16)


def test_parallel_tempering_rule_known_answers():
    """paratemp-MC/paratemp.f90:84-119: equal energies always swap (delta = 0,
    exp(0) = 1 > u), delta > 0 always swaps, unequal sizes never swap, and the
    starting pair alternates with the round parity."""
    kT = [1.0, 2.0, 3.0, 4.0, 5.0]
    sizes = [(8, 8)] * 5
    E = [0.0] * 5
    img, acc = O.pt_round(kT, range(5), E, sizes, 0, seed=1)
    assert img == [1, 0, 3, 2, 4] and acc == [0, 2]
    img, acc = O.pt_round(kT, range(5), E, sizes, 1, seed=1)
    assert img == [0, 2, 1, 4, 3] and acc == [1, 3]
    # colder slot holds the higher energy: (1/kT2 - 1/kT1) < 0, (E2 - E1) < 0, delta > 0
    img, acc = O.pt_round(kT, range(5), [5.0, 1.0, 5.0, 1.0, 0.0], sizes, 0, seed=1)
    assert acc == [0, 2]
    img, acc = O.pt_round(kT, range(5), E, [(8, 8), (9, 8), (8, 8), (8, 8), (8, 9)], 1, seed=1)
    assert acc == [] and img == [0, 1, 2, 3, 4]


def test_parallel_tempering_acceptance_rate():
    """For delta = -1 the swap is accepted with probability e^-1."""
    kT = [1.0, 0.5]          # 1/kT2 - 1/kT1 = 1
    E = [0.0, -1.0]          # E2 - E1 = -1  ->  delta = -1
    n = 20000
    hits = sum(len(O.pt_round(kT, [0, 1], E, [(4, 4)] * 2, 2 * r, seed=9)[1]) for r in range(n))
    p = np.exp(-1.0)
    assert abs(hits / n - p) < 4 * np.sqrt(p * (1 - p) / n)
    u = [O.pt_uniform(9, 0, r) for r in range(1000)]
    assert 0.0 <= min(u) and max(u) < 1.0 and len(set(u)) == 1000


def test_torch_sib_restatement_matches_oracle():
    """The float64 torch restatement used for the autograd checks follows the
    oracle's SIB trajectory (same couplings, field map and noise-free dynamics)."""
    import torch

    from matjes_b200.deck import random_sphere
    from tests import sib_torch_reference as R

    deck = square_film((8, 6, 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.5)
    n = deck.nsites
    m0 = random_sphere(n, 3)
    b = np.tile([0.0, 0.0, 0.5], (n, 1))
    A = R.unit_matrices(deck)
    terms = torch.tensor([1e-3, 0.3e-3, -0.1e-3], dtype=torch.float64)
    mt = R.trajectory(torch.tensor(m0), terms, torch.tensor(b), A, R.zeeman_coefficient(deck), 50, 0.1, 0.2)
    mo = m0.copy()
    O.Model(deck).run(mo, 50, integrator="sib", timestep=0.1, alpha=0.2)
    assert np.abs(mt.numpy() - mo).max() < 1e-12
