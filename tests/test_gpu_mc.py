"""Metropolis Monte Carlo on the device (mj_mc_sweeps) against the oracle.

The device moves the sites colour by colour with Philox draws keyed by (site,
sweep); the oracle's orc_mc_sweeps makes the same moves in the same colour
order, so the two chains agree move by move (states to rounding, acceptance
counts exactly).  The statistical tests hold the device chain to the
reference's parallel-tempering log (tests/serial/PTMC/EM.dat) and to the
Langevin function of a paramagnet."""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ptmc_ising_square20.json")))
KB = 8.6173324e-5


def batch_sem(x, nb=20):
    b = np.asarray(x)[: len(x) // nb * nb].reshape(nb, -1).mean(1)
    return b.std(ddof=1) / math.sqrt(nb)


def _decks():
    import matjes_b200 as mj

    return {
        "square": mj.square_film((24, 16, 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.5),
        "triangular": mj.triangular((18, 12)),
        "cubic": mj.square_film((8, 8, 4), Jv=1e-3, Dv=0.2e-3, Kv=0.05e-3, Bz=0.3, periodic=(1, 1, 1), a=0.25,
                                med_z=-0.3),
    }


@pytest.mark.parametrize("name", ["square", "triangular", "cubic"])
@pytest.mark.parametrize("proposal", ["sphere", "ising", "underrelax", "overrelax"])
def test_chain_equals_the_oracle_move_by_move(name, proposal):
    import torch

    import matjes_b200 as mj
    from matjes_b200.montecarlo import SAMPLING, MetropolisMC

    deck = _decks()[name]
    ham = mj.Hamiltonian(deck)
    mod = O.Model(deck)
    if name == "square":  # a site-dependent field through the plan's field map
        rng = np.random.default_rng(8)
        b = rng.normal(0.0, 0.5, (deck.ncell, 3))
        ham.set_bfield(b)
        mod.set_bfield(b)
    m0 = mj.random_sphere(deck.nsites, 17)
    m = torch.tensor(m0.T.copy(), device="cuda")
    T = 25.0
    chain = MetropolisMC(ham, proposal, cone=0.7, seed=0x5EED1234ABCD, stream_id=5, adapt_cone=True)
    E, Mg, acc = chain.sweeps(m, 12, T)
    E2, Mg2, acc2 = chain.sweeps(m, 5, T)  # a second call continues the chain (sweep counter, cone)
    torch.cuda.synchronize()
    mo = m0.copy()
    st = O.MC(temperature=T, cone=0.7, proposal=SAMPLING[proposal], adapt_cone=1, seed=0x5EED1234ABCD, stream_id=5,
              sweep0=0)
    Eo, Mgo, acco = O.mc_sweeps(mod, mo, st, 12, chain.colors, deck.L)
    Eo2, Mgo2, acco2 = O.mc_sweeps(mod, mo, st, 5, chain.colors, deck.L)
    assert (acc, acc2) == (acco, acco2) and acc > 0
    assert chain.p.accepted_total == st.accepted_total and chain.p.proposed_total == st.proposed_total == 17 * deck.nsites
    assert chain.p.sweep0 == st.sweep0 == 17 and chain.cone == st.cone
    assert np.abs(m.cpu().numpy().T - mo).max() < 1e-11
    scale = np.abs(Eo).max()
    assert np.abs(torch.cat([E, E2]).cpu().numpy() - np.concatenate([Eo, Eo2])).max() <= 1e-11 * scale
    assert np.abs(torch.cat([Mg, Mg2]).cpu().numpy() - np.concatenate([Mgo, Mgo2])).max() <= 1e-9
    # the colourings chosen: checkerboards for square and cubic nearest neighbours, (x + 3y) mod 9 for three triangular shells
    assert chain.colors == {"square": (2, 1, 0, 1), "cubic": (2, 1, 1, 1), "triangular": (9, 3, 0, 1)}[name]


@pytest.mark.parametrize("name", ["square", "triangular", "cubic"])
def test_tracked_totals_follow_the_recomputed_ones(name):
    """track_totals: the energy and summed spins of the call's start updated by
    every accepted move (track_val) equal the recomputed ones to rounding; the
    moves themselves do not change."""
    import torch

    import matjes_b200 as mj
    from matjes_b200.montecarlo import MetropolisMC

    deck = _decks()[name]
    ham = mj.Hamiltonian(deck)
    m0 = mj.random_sphere(deck.nsites, 5)
    out = {}
    for track in (False, True):
        m = torch.tensor(m0.T.copy(), device="cuda")
        ch = MetropolisMC(ham, "sphere", cone=0.8, seed=21, stream_id=2, adapt_cone=True, track_totals=track)
        E1, M1, a1 = ch.sweeps(m, 30, 12.0)
        E2, M2, a2 = ch.sweeps(m, 20, 40.0)
        out[track] = (m.cpu().numpy(), torch.cat([E1, E2]).cpu().numpy(), torch.cat([M1, M2]).cpu().numpy(), a1 + a2)
    (m_a, E_a, M_a, acc_a), (m_b, E_b, M_b, acc_b) = out[False], out[True]
    assert np.array_equal(m_a, m_b) and acc_a == acc_b
    assert np.abs(E_b - E_a).max() <= 1e-12 * np.abs(E_a).max()
    assert np.abs(M_b - M_a).max() <= 1e-10 * deck.nsites


def test_zero_temperature_and_unchanged_counter_streams():
    """At T = 0 only moves that lower the energy are taken; replicas on other
    stream ids draw other numbers."""
    import torch

    import matjes_b200 as mj
    from matjes_b200.montecarlo import MetropolisMC

    deck = mj.triangular((24, 24))
    ham = mj.Hamiltonian(deck)
    m0 = mj.random_sphere(deck.nsites, 3)
    ends = []
    for sid in (0, 1):
        m = torch.tensor(m0.T.copy(), device="cuda")
        E, _, acc = MetropolisMC(ham, "sphere", cone=0.4, seed=9, stream_id=sid, adapt_cone=False).sweeps(m, 40, 0.0)
        e = E.cpu().numpy()
        assert np.all(np.diff(e) <= 1e-15 * abs(e[0])) and acc > 0
        ends.append(m.cpu().numpy())
    assert np.abs(ends[0] - ends[1]).max() > 1e-3


def test_device_chain_reproduces_the_reference_ptmc_log():
    """Ising flips on the PTMC deck (20 x 20 square, J_1 = 0.5 meV) at each of
    the log's 40 temperatures: the mean energy per site within 4.5 standard
    errors of tests/serial/PTMC/EM.dat (the log's E_err / 10 from its 100
    measurements, ours from batch means over 2000 sweeps), the ordered
    magnetisation below 20 K."""
    import torch

    import matjes_b200 as mj
    from matjes_b200.montecarlo import MetropolisMC

    g = GOLD["deck"]
    deck = mj.square_film(tuple(g["L"]), Jv=g["J1"], Dv=0.0, Kv=g["K_z"], Bz=0.0, mu_s=g["mu_s"],
                          periodic=tuple(g["periodic"]))
    ham = mj.Hamiltonian(deck)
    N = deck.nsites
    for i, row in enumerate(GOLD["rows"]):
        T, E_gold, E_sd = row[0], row[1], row[2]
        m = torch.zeros((3, N), dtype=torch.float64, device="cuda")
        m[2] = 1.0
        chain = MetropolisMC(ham, "ising", seed=77, stream_id=i)
        E, Mg, _ = chain.sweeps(m, 2500, T)
        e = E[500:].cpu().numpy() / N
        tol = 4.5 * math.hypot(batch_sem(e), E_sd / math.sqrt(g["measurements"])) + 1e-12
        assert abs(e.mean() - E_gold) <= tol, (T, e.mean(), E_gold, tol)
        if T < 20.0:
            mz = Mg[500:, 2].cpu().numpy() / N
            assert abs(mz.mean() - row[4]) <= 4.0 * math.hypot(batch_sem(mz), 0.001) + 2e-4, (T, mz.mean(), row[4])
    assert chain.colors == (2, 1, 0, 1)


def test_paramagnet_follows_the_langevin_function():
    import torch

    import matjes_b200 as mj
    from matjes_b200.deck import Deck, square_areal
    from matjes_b200.montecarlo import MetropolisMC

    mu, B, T = 2.0, 3.0, 10.0
    deck = Deck(L=(16, 16, 1), periodic=(1, 1, 0), areal=square_areal(), atoms=[((0, 0, 0), 1, mu)], J=[], D=[],
                K=[], B_ext=(0.0, 0.0, B))
    ham = mj.Hamiltonian(deck)
    m = torch.zeros((3, deck.nsites), dtype=torch.float64, device="cuda")
    m[0] = 1.0
    _, Mg, _ = MetropolisMC(ham, "sphere", cone=math.pi, seed=1, adapt_cone=False).sweeps(m, 3000, T)
    mz = Mg[200:, 2].cpu().numpy() / deck.nsites
    x = mu * 5.78838180661e-5 * B / (KB * T)
    want = 1.0 / math.tanh(x) - 1.0 / x
    assert abs(mz.mean() - want) <= 5.0 * batch_sem(mz, 50)


def test_montecarlo_run_writes_the_thermodynamics(tmp_path):
    """The temperature loop of MonteCarlo.f90 (relaxation, T_auto sweeps per
    measurement) on the PTMC deck, and its EM.dat."""
    import torch

    import matjes_b200 as mj
    from matjes_b200.montecarlo import MCInput, montecarlo_run, thermo_print

    g = GOLD["deck"]
    deck = mj.square_film(tuple(g["L"]), Jv=g["J1"], Dv=0.0, Kv=g["K_z"], Bz=0.0, mu_s=g["mu_s"],
                          periodic=tuple(g["periodic"]))
    ham = mj.Hamiltonian(deck)
    m = torch.zeros((3, deck.nsites), dtype=torch.float64, device="cuda")
    m[2] = 1.0
    inp = MCInput(N_relaxation=200, T_relax=1, T_auto=2, Total_MC_Steps=1500, sampling="ising")
    rows = [GOLD["rows"][k] for k in (6, 14, 30)]
    out = montecarlo_run(ham, m, inp, [r[0] for r in rows], seed=4)
    for r, tv in zip(rows, out):
        assert abs(tv.E - r[1]) <= 4.5 * math.hypot(tv.E_err / math.sqrt(1500) * 3.0, r[2] / 10.0)
        assert tv.C > 0
    p = tmp_path / "EM.dat"
    thermo_print(str(p), out)
    assert len(p.read_text().splitlines()) == 4


def test_unsupported_plans_and_bad_arguments():
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi
    from matjes_b200.montecarlo import MetropolisMC

    dip = mj.square_film((8, 8, 2), Jv=1e-3, Dv=0.0, Kv=0.0, Bz=0.0, a=0.25, med_z=-0.3, dip=True)
    ham = mj.Hamiltonian(dip)
    m = torch.zeros((3, dip.nsites), dtype=torch.float64, device="cuda")
    m[2] = 1.0
    with pytest.raises(mj.MatjesError) as e:
        MetropolisMC(ham, "sphere").sweeps(m, 1, 10.0)
    assert e.value.status == _abi.MJ_ERR_UNSUPPORTED
    # periodic sizes 17 and 16 admit no linear colouring of the square stencil
    # (q must divide 17 and b 16 must be a multiple of q): the product one
    odd = mj.square_film((17, 16, 1), Jv=1e-3, Dv=0.0, Kv=0.0, Bz=0.0)
    ham2 = mj.Hamiltonian(odd)
    m2 = torch.zeros((3, odd.nsites), dtype=torch.float64, device="cuda")
    m2[2] = 1.0
    ch2 = MetropolisMC(ham2, "sphere")
    ch2.sweeps(m2, 1, 10.0)
    assert list(ch2.colors) == [17, 2, 1, 0]  # product colouring (x mod 17, y mod 2)
    sq = mj.square_film((8, 8, 1))
    ham3 = mj.Hamiltonian(sq)
    m3 = torch.zeros((3, sq.nsites), dtype=torch.float64, device="cuda")
    m3[2] = 1.0
    ch = MetropolisMC(ham3, "sphere")
    ch.p.proposal = 7
    with pytest.raises(mj.MatjesError) as e:
        ch.sweeps(m3, 1, 10.0)
    assert e.value.status == _abi.MJ_ERR_ARG
    with pytest.raises(mj.MatjesError):
        MetropolisMC(ham3, "sphere").sweeps(m3, 1, -1.0)
    with pytest.raises(ValueError):
        MetropolisMC(ham3, "heatbath")
    # nothing moved on the refused calls
    assert torch.equal(m3[2], torch.ones(sq.nsites, dtype=torch.float64, device="cuda"))


def test_reference_deck_directory_runs_the_monte_carlo(tmp_path):
    """run_montecarlo on an input directory: the PTMC deck in the reference's
    input format as `simulation metropolis` and as `simulation
    parallel-tempering`; EM.dat has one row per temperature, ascending, and the
    energies agree with the reference's log at those temperatures."""
    from matjes_b200 import reference_io as R

    deck_text = _MC_DECK
    for sim, extra in (("metropolis", ""), ("parallel-tempering", "n_sizerelax 1500\n")):
        d = tmp_path / sim
        d.mkdir()
        (d / "input").write_text(deck_text.replace("simulation metropolis", "simulation " + sim) + extra)
        m0 = np.zeros((400, 3))
        m0[:, 2] = 1.0
        R.write_order_file(str(d / "magnetic_init.dat"), m0)
        rows = R.run_montecarlo(str(d), seed=3)
        lines = (d / "EM.dat").read_text().splitlines()
        assert len(rows) == 4 and len(lines) == 5
        Ts = [r.T for r in rows]
        assert Ts == sorted(Ts) and Ts[0] == pytest.approx(11.769230769, rel=1e-9)
        for tv in rows:
            ref = min(GOLD["rows"], key=lambda r: abs(r[0] - tv.T))
            assert abs(ref[0] - tv.T) < 1e-6
            # a few hundred correlated samples: within 6 of the log's sample deviations
            assert abs(tv.E - ref[1]) <= 6.0 * ref[2] + 1e-9, (sim, tv.T, tv.E, ref[1])


_MC_DECK = """simulation metropolis
Periodic_log .T. .T. .F.
lattice
1.0 0.0 0.0
0.0 1.0 0.0
0.0 0.0 1.0
Nsize 20 20 1
atomtypes 1
Fe 3.0 0.0 1.0 F
atoms 1
Fe 0.0 0.0 0.0
magnetic_J
1 1 1 0.5d-3
magnetic_anisotropy
1 0.0 0.0 1.0 5.0d-7
Tini 11.769230769230769
Tfin 16.384615384615383
n_Tsteps 4
n_relaxation 100
T_relax 1
T_auto 2
Total_MC_Steps 600
cone 1.0
ising .T.
"""


@pytest.mark.parametrize("L,colors", [((17, 17), [17, 1, 0, 1]), ((13, 26), [13, 1, 0, 1])])
def test_prime_periodic_sizes_take_as_many_colours(L, colors):
    """A periodic size p prime admits only colourings of p colours along it:
    the chain then moves colour by colour as the oracle does, move by move."""
    import torch

    import matjes_b200 as mj
    from matjes_b200.montecarlo import SAMPLING, MetropolisMC

    deck = mj.square_film((L[0], L[1], 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.5)
    ham = mj.Hamiltonian(deck)
    m0 = mj.random_sphere(deck.nsites, 3)
    m = torch.tensor(m0.T.copy(), device="cuda")
    chain = MetropolisMC(ham, "sphere", cone=0.6, seed=11, stream_id=2, adapt_cone=False)
    E, Mg, acc = chain.sweeps(m, 6, 30.0)
    torch.cuda.synchronize()
    assert list(chain.colors) == colors
    mo = m0.copy()
    st = O.MC(temperature=30.0, cone=0.6, proposal=SAMPLING["sphere"], adapt_cone=0, seed=11, stream_id=2, sweep0=0)
    Eo, Mgo, acco = O.mc_sweeps(O.Model(deck), mo, st, 6, chain.colors, deck.L)
    assert acc == acco > 0
    assert np.abs(m.cpu().numpy().T - mo).max() < 1e-11
    assert np.abs(E.cpu().numpy() - Eo).max() <= 1e-11 * np.abs(Eo).max()
