"""Metropolis Monte Carlo: the oracle's chains pinned to the reference's PTMC
golden log and to analytic results, and the host-side thermodynamics (CPU)."""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ptmc_ising_square20.json")))
KB = 8.6173324e-5


def ptmc_deck():
    from matjes_b200.deck import square_film

    g = GOLD["deck"]
    return square_film(tuple(g["L"]), Jv=g["J1"], Dv=0.0, Kv=g["K_z"], Bz=0.0, mu_s=g["mu_s"],
                       periodic=tuple(g["periodic"]))


def batch_sem(x, nb=20):
    b = np.asarray(x)[: len(x) // nb * nb].reshape(nb, -1).mean(1)
    return b.std(ddof=1) / math.sqrt(nb)


def test_ptmc_deck_ground_state_energy():
    """-4 J_1 + K per site in the +z state: the log's low-temperature E_av."""
    mod = O.Model(ptmc_deck())
    m = np.zeros((400, 3))
    m[:, 2] = 1.0
    assert mod.energy(m) / 400 == pytest.approx(GOLD["rows"][0][1], abs=1e-15)


def test_random_site_chain_reproduces_the_reference_ptmc_log():
    """The reference's move order (choose_spin, Ising flips, MCstep acceptance)
    against tests/serial/PTMC/EM.dat: at each of the 40 temperatures the mean
    energy per site within 4.5 standard errors (the log's from its 100
    measurements, E_err / 10; ours from batch means over 2000 sweeps), and the
    ordered magnetisation below 20 K."""
    mod = O.Model(ptmc_deck())
    N = 400
    n_log = GOLD["deck"]["measurements"]
    for row in GOLD["rows"]:
        T, E_gold, E_sd = row[0], row[1], row[2]
        m = np.zeros((N, 3))
        m[:, 2] = 1.0
        st = O.MC(temperature=T, cone=1.0, proposal=1, adapt_cone=0, seed=20240607, stream_id=3, sweep0=0)
        E, Mg, _ = O.mc_random(mod, m, st, 2500)
        e = E[500:] / N
        tol = 4.5 * math.hypot(batch_sem(e), E_sd / math.sqrt(n_log)) + 1e-12
        assert abs(e.mean() - E_gold) <= tol, (T, e.mean(), E_gold, tol)
        if T < 20.0:
            mz = Mg[500:, 2] / N
            assert abs(mz.mean() - row[4]) <= 4.0 * math.hypot(batch_sem(mz), 0.001) + 2e-4, (T, mz.mean(), row[4])


def test_tracked_energy_equals_the_recomputed_total():
    """track_val's E_total (updated by each accepted dE) ends equal to H%energy:
    the single-site energy change is the change of the total, with DMI,
    anisotropy and field."""
    from matjes_b200.deck import random_sphere, square_film

    d = square_film((8, 6, 1), Jv=1e-3, Dv=0.4e-3, Kv=-0.2e-3, Bz=0.7)
    mod = O.Model(d)
    m = random_sphere(d.nsites, 4)
    for prop in (0, 1, 2, 3):
        st = O.MC(temperature=15.0, cone=0.8, proposal=prop, adapt_cone=1, seed=7, stream_id=0, sweep0=0)
        E, _, _ = O.mc_random(mod, m, st, 20)
        assert E[-1] == pytest.approx(mod.energy(m), rel=1e-11, abs=1e-14)
        assert np.allclose(np.linalg.norm(m, axis=1), 1.0, atol=1e-14)


def test_single_spin_in_a_field_follows_the_langevin_function():
    """One classical moment mu_s in B along z: <m_z> = coth(x) - 1/x,
    x = mu_s muB B / kT (full-sphere cone proposals), both move orders."""
    from matjes_b200.deck import Deck, square_areal

    mu, B, T = 2.0, 3.0, 10.0
    d = Deck(L=(1, 1, 1), periodic=(0, 0, 0), areal=square_areal(), atoms=[((0, 0, 0), 1, mu)], J=[], D=[], K=[],
             B_ext=(0.0, 0.0, B))
    mod = O.Model(d)
    x = mu * 5.78838180661e-5 * B / (KB * T)
    want = 1.0 / math.tanh(x) - 1.0 / x
    for order in ("random", "colour"):
        m = np.array([[1.0, 0.0, 0.0]])
        st = O.MC(temperature=T, cone=math.pi, proposal=0, adapt_cone=0, seed=11, stream_id=0, sweep0=0)
        if order == "random":
            _, Mg, _ = O.mc_random(mod, m, st, 200000)
        else:
            _, Mg, _ = O.mc_sweeps(mod, m, st, 200000, (2, 1, 1, 0), d.L)
        mz = Mg[1000:, 2]
        assert abs(mz.mean() - want) <= 5.0 * batch_sem(mz, 50), (order, mz.mean(), want)


def test_colour_order_samples_the_reference_distribution():
    """Sweeps colour by colour and the reference's random-site order give the
    same equilibrium averages (Heisenberg film with DMI, anisotropy and field,
    fixed cone)."""
    from matjes_b200.deck import square_film

    d = square_film((12, 12, 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.5)
    mod = O.Model(d)
    N = d.nsites
    res = {}
    for order in ("random", "colour"):
        m = np.zeros((N, 3))
        m[:, 2] = 1.0
        st = O.MC(temperature=8.0, cone=0.9, proposal=0, adapt_cone=0, seed=5, stream_id=1, sweep0=0)
        if order == "random":
            E, Mg, _ = O.mc_random(mod, m, st, 6000)
        else:
            E, Mg, _ = O.mc_sweeps(mod, m, st, 6000, (2, 1, 0, 1), d.L)  # checkerboard
        res[order] = (E[1000:] / N, Mg[1000:, 2] / N)
    (ea, ma), (eb, mb) = res["random"], res["colour"]
    assert abs(ea.mean() - eb.mean()) <= 4.5 * math.hypot(batch_sem(ea), batch_sem(eb))
    assert abs(ma.mean() - mb.mean()) <= 4.5 * math.hypot(batch_sem(ma), batch_sem(mb))


def test_zero_temperature_moves_never_raise_the_energy():
    from matjes_b200.deck import random_sphere, triangular

    d = triangular((12, 12))
    mod = O.Model(d)
    m = random_sphere(d.nsites, 2)
    st = O.MC(temperature=0.0, cone=0.5, proposal=0, adapt_cone=1, seed=3, stream_id=0, sweep0=0)
    E, _, acc = O.mc_sweeps(mod, m, st, 30, (3, 3, 1, 0), d.L)
    assert np.all(np.diff(E) <= 1e-15) and acc > 0
    # the adaptive cone stays inside [0.01, pi]
    assert 0.01 <= st.cone <= math.pi and st.sweep0 == 30


def test_site_colourings():
    sc, nc = O.mc_site_colours((4, 2, 1), (2, 1, 0, 1))
    assert nc == 2 and sc.tolist() == [0, 1, 0, 1, 1, 0, 1, 0]
    sc, nc = O.mc_site_colours((3, 2, 2), (3, 1, 2, 0))
    assert nc == 6 and sc.reshape(2, 2, 3)[1, 1].tolist() == [3, 4, 5] and sc[0] == 0


def test_temperature_grid_and_thermo_averages():
    from matjes_b200.montecarlo import temperatures, therm_set

    T = temperatures(1.0, 61.0, 40)
    np.testing.assert_allclose(T, [r[0] for r in GOLD["rows"]], rtol=0, atol=5e-9)
    assert temperatures(2.0, 9.0, 1).tolist() == [2.0]
    np.testing.assert_allclose(temperatures(1.0, 100.0, 3, geometric=True), [1.0, 10.0, 100.0])
    rng = np.random.default_rng(0)
    E = rng.normal(-3.0, 0.01, 10)
    M = rng.normal(0.0, 1.0, (10, 3))
    tv = therm_set(20.0, E, M, 50)
    kT = 20.0 * KB
    assert tv.E == pytest.approx(E.mean() / 50, rel=1e-14)
    assert tv.C == pytest.approx(E.var() / kT ** 2 / 50, rel=1e-8)
    assert tv.E_err == pytest.approx(E.std(ddof=1) / 50, rel=1e-8)
    np.testing.assert_allclose(tv.chi_M, M.var(0) / kT / 50, rtol=1e-8)
    np.testing.assert_allclose(tv.M_err, M.std(0, ddof=1) / 50, rtol=1e-8)
    # the log's C and E_err columns are these estimators of its 100 measurements
    n = GOLD["deck"]["measurements"]
    for r in GOLD["rows"][5:]:
        assert r[3] == pytest.approx(r[2] ** 2 * 400 / (r[0] * KB) ** 2 * (n - 1) / n, rel=1e-7)


def test_em_dat_number_format(tmp_path):
    """(E20.10E3) of thermo_print: each token of the reference's log reproduced."""
    from matjes_b200.montecarlo import ThermVal, thermo_print
    from matjes_b200.reference_io import fortran_e

    for toks in GOLD["tokens"]:
        for t in toks:
            assert fortran_e(float(t), 20, 10, 3).strip() == t
    rows = [ThermVal(24.07692308, -0.0016902, 9.898734742e-05, 0.9013778829, np.array([0.0, 0.0, 0.8812]),
                     np.zeros(3), np.zeros(3))]
    p = tmp_path / "EM.dat"
    thermo_print(str(p), rows)
    lines = p.read_text().splitlines()
    assert lines[0].startswith("# 1:T" + " " * 15 + "2:E_av")
    assert len(lines[1]) == 35 * 20 + 34 * 2
    vals = lines[1].split()
    assert len(vals) == 35 and vals[0] == "0.2407692308E+002" and vals[4] == "0.8812000000E+000"
