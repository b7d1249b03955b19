"""Parallel-tempering Monte Carlo on batched replicas (mj_batch_mc).

Every replica is a Metropolis chain of its own: without swaps it must equal
the oracle's chain of its lattice alone (stream stream_id + r, its field and
temperature) move by move.  With swaps the temperatures must follow the
reference's rule (paratemp-MC/paratemp.f90:84-119), restated by the oracle, on
the same energies; and the ladder run must reproduce the reference's own
parallel-tempering log (tests/serial/PTMC/EM.dat)."""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

KB = 0.000086173324
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ptmc_ising_square20.json")))


def batch_sem(x, nb=20):
    b = np.asarray(x)[: len(x) // nb * nb].reshape(nb, -1).mean(1)
    return b.std(ddof=1) / math.sqrt(nb)


def _square(sizes, Bz, Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3):
    import matjes_b200 as mj

    cell = mj.square_film((8, 8, 1), Jv=Jv, Dv=Dv, Kv=Kv, Bz=0.0)
    B = np.zeros((len(sizes), 3))
    B[:, 2] = Bz
    decks = [mj.square_film((lx, ly, 1), Jv=Jv, Dv=Dv, Kv=Kv, Bz=bz) for (lx, ly), bz in zip(sizes, Bz)]
    return cell, B, decks


@pytest.mark.parametrize("proposal", ["sphere", "ising", "overrelax"])
def test_replicas_are_the_oracle_chains_of_their_lattices(proposal):
    import matjes_b200 as mj
    from matjes_b200 import _abi
    from matjes_b200.montecarlo import SAMPLING

    sizes = [(16, 16), (24, 16), (16, 34), (8, 8), (40, 4)]
    Bz = [0.3, 0.0, 1.1, 2.0, 0.6]
    T = [5.0, 15.0, 30.0, 60.0, 0.0]
    cell, B, decks = _square(sizes, Bz)
    batch = mj.ReplicaBatch(cell, sizes, B, T)
    m0 = [mj.random_sphere(d.nsites, 40 + r) for r, d in enumerate(decks)]
    batch.upload(np.concatenate(m0))
    seed, sid, spr, nr = 0xABCDEF12345, 3, 4, 3
    p = _abi.McParams(0.0, 0.6, SAMPLING[proposal], 1, seed, sid, 0, 0, 0, 0, 0)
    E, M, S = batch.monte_carlo(p, nr, spr, swap=False)
    E, M, S = E.cpu().numpy(), M.cpu().numpy(), S.cpu().numpy()
    out = batch.download()
    cone, acc, prop = batch.mc_state()
    assert batch.mc_colors == (2, 1, 0, 1) and p.sweep0 == nr * spr and p.round0 == 0
    for r, d in enumerate(decks):
        m = m0[r].copy()
        st = O.MC(temperature=T[r], cone=0.6, proposal=SAMPLING[proposal], adapt_cone=1, seed=seed, stream_id=sid + r,
                  sweep0=0)
        Eo, Mo, _ = O.mc_sweeps(O.Model(d), m, st, nr * spr, batch.mc_colors, d.L)
        a, b = batch.offsets[r], batch.offsets[r + 1]
        assert np.abs(out[a:b] - m).max() < 1e-11, r
        assert acc[r] == st.accepted_total and prop[r] == st.proposed_total == nr * spr * d.nsites
        assert cone[r] == st.cone
        np.testing.assert_allclose(E[:, r], Eo[spr - 1::spr], rtol=1e-11, atol=1e-14)
        np.testing.assert_allclose(M[:, r], Mo[spr - 1::spr], rtol=0, atol=1e-9)
    # without swaps every replica keeps its slot
    assert (S == S[0]).all()


def test_swap_rounds_follow_the_reference_rule():
    import matjes_b200 as mj
    from matjes_b200 import _abi

    n = 10
    sizes = [(12, 12)] * 4 + [(16, 12)] + [(12, 12)] * (n - 5)
    T = list(6.0 + 1.2 * np.arange(n))[::-1]  # descending: the ladder order is not the replica order
    cell, B, decks = _square(sizes, [0.4] * n)
    batch = mj.ReplicaBatch(cell, sizes, B, T)
    m0 = [mj.random_sphere(d.nsites, 7 + r) for r, d in enumerate(decks)]
    batch.upload(np.concatenate(m0))
    seed, spr, nr = 2024, 3, 8
    p = _abi.McParams(0.0, 0.5, _abi.MJ_MC_CONE, 0, seed, 0, 0, 0, 0, 0, 0)
    E, M, S = batch.monte_carlo(p, nr, spr, swap=True)
    E, S = E.cpu().numpy(), S.cpu().numpy()
    order = sorted(range(n), key=lambda r: T[r])
    kT_slot = [T[r] * KB for r in order]
    image = list(order)
    ms = [m.copy() for m in m0]
    sts = [O.MC(temperature=0.0, cone=0.5, proposal=0, adapt_cone=0, seed=seed, stream_id=r, sweep0=0)
           for r in range(n)]
    models = [O.Model(d) for d in decks]
    nswap = 0
    for k in range(nr):
        slot = np.empty(n, np.int32)
        for l, r in enumerate(image):
            slot[r] = l
        assert np.array_equal(S[k], slot), k
        Eo = np.empty(n)
        for r in range(n):
            sts[r].temperature = kT_slot[slot[r]] / KB
            Eo[r] = O.mc_sweeps(models[r], ms[r], sts[r], spr, batch.mc_colors, decks[r].L)[0][-1]
        np.testing.assert_allclose(E[k], Eo, rtol=1e-11)
        image, acc = O.pt_round(kT_slot, image, Eo, sizes, k, seed)
        nswap += len(acc)
    T_gpu, acc_gpu = batch.temperatures()
    for l, r in enumerate(image):
        assert T_gpu[r] == pytest.approx(kT_slot[l] / KB, rel=1e-13)
    assert acc_gpu.sum() == nswap > 0
    assert T_gpu[4] == pytest.approx(T[4], rel=1e-13)  # the odd-sized replica never swaps
    out = batch.download()
    for r in range(n):
        assert np.abs(out[batch.offsets[r]:batch.offsets[r + 1]] - ms[r]).max() < 1e-11
    assert p.round0 == nr


def test_ladder_run_reproduces_the_reference_ptmc_log():
    """The reference's parallel-tempering test (40 replicas of the 20 x 20
    Ising square at 1 .. 61 K, Ising sampling from +z) as a batch: after 300
    unmeasured rounds, 3000 measured rounds of one sweep; the mean energy per
    site of every ladder temperature within 4.5 standard errors of the log."""
    import matjes_b200 as mj
    from matjes_b200 import _abi
    from matjes_b200.montecarlo import MCInput, parallel_tempering_run

    g = GOLD["deck"]
    Ts = [r[0] for r in GOLD["rows"]]
    n = len(Ts)
    cell = mj.square_film((20, 20, 1), Jv=g["J1"], Dv=0.0, Kv=g["K_z"], Bz=0.0, mu_s=g["mu_s"],
                          periodic=tuple(g["periodic"]))
    batch = mj.ReplicaBatch(cell, [(20, 20)] * n, np.zeros((n, 3)), Ts)
    m0 = np.zeros((400 * n, 3))
    m0[:, 2] = 1.0
    batch.upload(m0)
    relax = _abi.McParams(0.0, 1.0, _abi.MJ_MC_ISING, 0, 99, 0, 0, 0, 0, 0, 0)
    batch.monte_carlo(relax, 300, 1, swap=True, record=False)
    inp = MCInput(n_sizerelax=3000, T_auto=1, sampling="ising", cone=1.0)
    rows, (E, M, S) = parallel_tempering_run(batch, inp, seed=1234, stream_id=1000, return_series=True)
    assert [r.T for r in rows] == pytest.approx(Ts, rel=1e-13)
    assert E.shape == (3000, n) and all(sorted(s_) == list(range(n)) for s_ in S.tolist())
    for l, (tv, ref) in enumerate(zip(rows, GOLD["rows"])):
        e = E[S == l] / 400  # the energies measured at ladder temperature l, in round order
        assert tv.E == pytest.approx(e.mean(), rel=1e-12)
        tol = 4.5 * math.hypot(batch_sem(e, 10), ref[2] / math.sqrt(g["measurements"])) + 1e-12
        assert abs(tv.E - ref[1]) <= tol, (tv.T, tv.E, ref[1], tol)
    _, acc = batch.temperatures()
    assert acc.sum() > 0
