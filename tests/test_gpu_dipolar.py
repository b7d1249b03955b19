"""FFT dipolar (cuFFT + hand-written pad / pointwise / fused unpack) against the oracle."""
import numpy as np
import pytest

from conftest import scalar_rel_err, site_rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _film(L, periodic, **kw):
    import matjes_b200 as mj

    return mj.square_film(L, periodic=periodic, a=0.25, med_z=-0.3, dip=True, **kw)


@pytest.mark.parametrize("L,periodic", [((16, 16, 4), (1, 1, 0)), ((6, 5, 4), (0, 0, 0)), ((8, 8, 8), (1, 1, 1)),
                                        ((12, 10, 3), (1, 0, 0))])
def test_dipolar_field_energy_match_oracle(L, periodic):
    import matjes_b200 as mj

    deck = _film(L, periodic, Jv=1e-3, Dv=0.15e-3, Kv=-0.02e-3, Bz=0.2)
    ham = mj.Hamiltonian(deck)
    M = O.Model(deck)
    m = mj.random_sphere(deck.nsites, 8)
    B, e = ham.get_eff_field(m, with_energy=True)
    Bo, eo = M.field(m)
    assert site_rel_err(B, Bo) < 1e-12
    assert scalar_rel_err(e, eo) < 1e-12
    assert abs(ham.energy(m) - M.energy(m)) <= 1e-12 * abs(M.energy(m))


def test_dipolar_only_field_against_explicit_pair_sum_open_cube():
    import matjes_b200 as mj

    deck = _film((6, 6, 5), (0, 0, 0), Jv=0.0, Dv=0.0, Kv=0.0, Bz=0.0)
    ham = mj.Hamiltonian(deck)
    m = mj.random_sphere(deck.nsites, 3)
    B = ham.get_eff_field(m)
    Bx = O.Model(deck).dipolar_explicit(m)
    assert np.abs(B - Bx).max() < 1e-12 * np.abs(Bx).max()


@pytest.mark.parametrize("integrator", ["sib", "heun"])
def test_dipolar_trajectory(integrator):
    import matjes_b200 as mj

    deck = _film((16, 16, 4), (1, 1, 0), Jv=1e-3, Dv=0.15e-3, Kv=-0.02e-3, Bz=0.2)
    m0 = mj.random_sphere(deck.nsites, 4)
    dyn = dict(integrator=integrator, timestep=0.1, alpha=0.1, temperature=0.0)
    m = m0.copy()
    mj.SpinDynamics(mj.Hamiltonian(deck), **dyn).run(m, 100)
    mo = m0.copy()
    O.Model(deck).run(mo, 100, **dyn)
    assert np.abs(m - mo).max() < 1e-9


def test_zero_padded_grid_matches_the_explicit_pair_sum():
    """dip = 2 (every axis longer than one cell zero-padded to 2 L) on a film
    periodic in plane: the device field equals the oracle's explicit pair sum,
    and the whole field (all terms) the oracle's to 1e-12."""
    import matjes_b200 as mj

    deck = mj.square_film((8, 6, 3), Jv=0.0, Dv=0.0, Kv=0.0, Bz=0.0, periodic=(1, 1, 0), a=0.25, dip=2)
    m = mj.random_sphere(deck.nsites, 9)
    B = mj.Hamiltonian(deck).get_eff_field(m)
    Bx = O.Model(deck).dipolar_explicit(m)
    assert np.abs(B - Bx).max() < 1e-12 * np.abs(Bx).max()
    full = mj.square_film((16, 16, 4), Jv=1e-3, Dv=0.15e-3, Kv=-0.02e-3, Bz=0.2, periodic=(1, 1, 0), a=0.25,
                          med_z=-0.3, dip=2)
    m = mj.random_sphere(full.nsites, 10)
    B, e = mj.Hamiltonian(full).get_eff_field(m, with_energy=True)
    Bo, eo = O.Model(full).field(m)
    assert site_rel_err(B, Bo) < 1e-12
    assert scalar_rel_err(e, eo) < 1e-12


@pytest.mark.parametrize("dip", [1, 2])
def test_full_size_film_field_and_sib_steps(dip):
    """The dipolar workload at its full size (128 x 128 x 16 simple cubic, a =
    0.25 nm, periodic in plane, open along z; J + D + K + Bz = 0.2 T + FFT
    dipolar, mu_s = 2): on the reference's grid (dip = 1, 128 x 128 x 32) and
    on the fully zero-padded one (dip = 2, 256 x 256 x 32) the field and the
    per-site energies equal the oracle's to 1e-12, and 20 SIB steps with
    Philox noise at 5 K stay within 1e-9 of the oracle's."""
    import matjes_b200 as mj

    w = mj.workload("film128x16_dipolar")
    deck = w["deck"]
    deck.dip = dip
    ham = mj.Hamiltonian(deck)
    M = O.Model(deck)
    assert M.nrep() == ((128, 128, 32) if dip == 1 else (256, 256, 32))
    m0 = w["m0"]
    B, e = ham.get_eff_field(m0, with_energy=True)
    Bo, eo = M.field(m0)
    assert site_rel_err(B, Bo) < 1e-12
    assert scalar_rel_err(e, eo) < 1e-12
    dyn = dict(w["dyn"])
    dyn.pop("steps")
    m = m0.copy()
    mj.SpinDynamics(ham, **dyn).run(m, 20)
    mo = m0.copy()
    M.run(mo, 20, **dyn)
    assert np.abs(m - mo).max() < 1e-9
    assert np.abs(np.linalg.norm(m, axis=1) - 1.0).max() < 1e-13


@pytest.mark.parametrize("L,periodic,dip", [((16, 16, 4), (1, 1, 0), 1), ((8, 8, 8), (1, 1, 1), 1),
                                            ((6, 5, 4), (0, 0, 0), 1), ((16, 16, 4), (1, 1, 0), 2),
                                            ((12, 10, 2), (1, 0, 0), 1)])
def test_fused_z_convolution_equals_the_cufft_route(L, periodic, dip):
    """z grids of 16, 8, 8, 8 and 4 planes: the fused z transforms and product
    (lane FFTs, K_F per column) give the field and energies of the cuFFT z
    transforms with the separate product to 1e-13."""
    import matjes_b200 as mj
    from matjes_b200 import _abi

    deck = _film(L, periodic, Jv=1e-3, Dv=0.15e-3, Kv=-0.02e-3, Bz=0.2)
    deck.dip = dip
    m = mj.random_sphere(deck.nsites, 12)
    out = []
    for zconv in (1, 0):
        ham = mj.Hamiltonian(deck)
        _abi.check(_abi.lib.mj_plan_set_option(ham.plan, _abi.MJ_OPT_DIP_ZCONV, zconv))
        out.append(ham.get_eff_field(m, with_energy=True))
    (B1, e1), (B0, e0) = out
    assert site_rel_err(B1, B0) < 1e-13
    assert scalar_rel_err(e1, e0) < 1e-13


@pytest.mark.parametrize("integrator", ["sib", "heun", "euler"])
def test_pad_written_by_the_steps_is_never_stale(integrator):
    """Within a step sequence the step kernels also write the dipolar term's
    padded input grid; a call that follows, after the caller replaced the
    spins, must see the new spins: 6 steps, new spins, 6 more steps, each part
    against the oracle (and a field evaluation in between)."""
    import torch

    import matjes_b200 as mj

    deck = _film((16, 16, 4), (1, 1, 0), Jv=1e-3, Dv=0.15e-3, Kv=-0.02e-3, Bz=0.2)
    ham = mj.Hamiltonian(deck)
    M = O.Model(deck)
    dyn = dict(integrator=integrator, timestep=0.1, alpha=0.1, temperature=0.0)
    sd = mj.SpinDynamics(ham, **dyn)
    m0 = mj.random_sphere(deck.nsites, 31)
    m = torch.tensor(m0.T.copy(), device="cuda")
    sd.run(m, 6)
    mo = m0.copy()
    M.run(mo, 6, **dyn)
    assert np.abs(m.cpu().numpy().T - mo).max() < 1e-11
    m1 = mj.random_sphere(deck.nsites, 32)
    m.copy_(torch.tensor(m1.T.copy(), device="cuda"))
    B = ham.get_eff_field(m1)
    Bo, _ = M.field(m1)
    assert site_rel_err(B, Bo) < 1e-12
    sd.run(m, 6)
    mo = m1.copy()
    M.run(mo, 6, **dyn)
    assert np.abs(m.cpu().numpy().T - mo).max() < 1e-11
