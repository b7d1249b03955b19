"""Batched replicas (mj_batch_*) against single-lattice runs and the oracle.

Every replica of a batch must follow the trajectory of its own lattice run
alone: the same SIB arithmetic, its own applied field and temperature, Philox
noise on stream stream_id + r with its local site indices.  The
parallel-tempering rounds must permute the temperatures exactly as the
reference's rule (paratemp-MC/paratemp.f90:84-119), restated by the oracle,
does on the same energies and draws.  Graph replay, tile variants and
persistent grid sizes must not change a bit of the result.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

KB = 0.000086173324
TRAJ_TOL = 1e-9     # max |dm| against the oracle after the steps below
E_TOL = 1e-12       # relative energy tolerance


def _square_batch(sizes, Bz, T, periodic=(1, 1, 0)):
    import matjes_b200 as mj

    cell = mj.square_film((8, 8, 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.0, periodic=periodic)
    B = np.zeros((len(sizes), 3))
    B[:, 2] = Bz
    decks = [mj.square_film((lx, ly, 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=bz, periodic=periodic)
             for (lx, ly), bz in zip(sizes, Bz)]
    return cell, B, decks


def _tri_batch(sizes, Bz):
    import matjes_b200 as mj

    cell = mj.triangular((8, 8), Bz=0.0)
    B = np.zeros((len(sizes), 3))
    B[:, 2] = Bz
    decks = [mj.triangular((lx, ly), Bz=bz) for (lx, ly), bz in zip(sizes, Bz)]
    return cell, B, decks


CASES = {
    # uneven sizes, sides not multiples of the 32 x 16 tile, one tiny replica
    "square_mixed": lambda: _square_batch([(32, 32), (48, 40), (17, 23), (64, 64), (5, 7)],
                                          [0.5, 1.3, 0.0, 2.0, 0.7], [0.0, 5.0, 10.0, 20.0, 40.0]),
    "square_open_x": lambda: _square_batch([(40, 24), (33, 33), (16, 64)], [0.2, 0.9, 1.7], [3.0, 0.0, 30.0],
                                           periodic=(0, 1, 0)),
    "triangular_3_shells": lambda: _tri_batch([(48, 32), (35, 29), (64, 16)], [1.0, 0.3, 1.6]),
}
TEMPS = {"square_mixed": [0.0, 5.0, 10.0, 20.0, 40.0], "square_open_x": [3.0, 0.0, 30.0],
         "triangular_3_shells": [10.0, 2.0, 25.0]}


def _initial(decks, seed):
    import matjes_b200 as mj

    return [mj.random_sphere(d.nsites, seed + r) for r, d in enumerate(decks)]


@pytest.mark.parametrize("case", sorted(CASES))
def test_batch_replicas_follow_their_own_runs(case):
    import matjes_b200 as mj

    cell, B, decks = CASES[case]()
    T = TEMPS[case]
    sizes = [d.L[:2] for d in decks]
    ms = _initial(decks, 11)
    batch = mj.ReplicaBatch(cell, sizes, B, T)
    batch.upload(np.concatenate(ms))
    nsteps, seed, stream0 = 60, 7, 3
    p = batch.params(timestep=0.1, alpha=0.5, noise="philox", seed=seed, stream_id=stream0)
    batch.step(p, nsteps)
    out = batch.download()
    E = batch.energies()
    for r, deck in enumerate(decks):
        dyn = dict(integrator="sib", timestep=0.1, alpha=0.5, temperature=T[r], noise="philox", seed=seed,
                   stream_id=stream0 + r)
        m_plain = ms[r].copy()
        mj.SpinDynamics(mj.Hamiltonian(deck), **dyn).run(m_plain, nsteps)
        mb = batch.replica(out, r)
        # same arithmetic as the single-lattice tiled kernels
        assert np.abs(mb - m_plain).max() <= 1e-13, (case, r)
        mo = ms[r].copy()
        O.Model(deck).run(mo, nsteps, stream=stream0 + r, **dyn)
        assert np.abs(mb - mo).max() < TRAJ_TOL, (case, r)
        assert np.abs(np.linalg.norm(mb, axis=1) - 1.0).max() < 1e-13
        Eo = O.Model(deck).energy(mb)
        assert abs(E[r] - Eo) <= E_TOL * abs(Eo), (case, r)


def test_batch_variants_and_grids_bitwise_equal():
    import matjes_b200 as mj

    cell, B, decks = CASES["square_mixed"]()
    m0 = np.concatenate(_initial(decks, 5))
    ref = None
    for v in range(5):
        for bps in (1, 3, 8, 32):
            batch = mj.ReplicaBatch(cell, [d.L[:2] for d in decks], B, TEMPS["square_mixed"])
            batch.set_config(v, bps)
            batch.upload(m0)
            batch.step(batch.params(seed=2, noise="philox"), 12)
            out = batch.download()
            if ref is None:
                ref = out
            assert np.array_equal(out, ref), (v, bps)
            batch.close()


def _ladder(T):
    order = sorted(range(len(T)), key=lambda r: T[r])
    return [T[r] * KB for r in order], order


def test_parallel_tempering_rounds_follow_the_reference_rule():
    import matjes_b200 as mj

    # equal sizes on most ladder neighbours, temperatures close enough that the
    # Metropolis draw decides some pairs; one odd size that must never swap
    sizes = [(8, 8)] * 9 + [(12, 8)] + [(8, 8)] * 6
    n = len(sizes)
    T = list(60.0 + 1.5 * np.arange(n))
    Bz = np.linspace(0.0, 0.2, n)
    cell, B, _ = _square_batch(sizes, Bz, T)
    m0 = mj.random_sphere(sum(a * b for a, b in sizes), 21)
    K, seed = 10, 77
    p_args = dict(timestep=0.1, alpha=0.5, noise="philox", seed=seed)

    swap = mj.ReplicaBatch(cell, sizes, B, T)
    swap.upload(m0)
    plain = mj.ReplicaBatch(cell, sizes, B, T)
    plain.upload(m0)
    ps, pp = swap.params(**p_args), plain.params(**p_args)

    kT_slot, image = _ladder(T)
    swap.step(ps, K, swap_every=K)          # round 1 after step K-1
    plain.step(pp, K)
    assert np.array_equal(swap.download(), plain.download())  # a swap leaves the spins alone
    E1 = plain.energies()
    image, acc1 = O.pt_round(kT_slot, image, E1, sizes, 1, seed)
    T_gpu, acc_gpu = swap.temperatures()
    T_pred = np.empty(n)
    for l, r in enumerate(image):
        T_pred[r] = kT_slot[l] / KB
    np.testing.assert_allclose(T_gpu, T_pred, rtol=1e-13)

    swap.step(ps, K, swap_every=K)          # round 2 on the swapped temperatures
    E2 = swap.energies()
    image, acc2 = O.pt_round(kT_slot, image, E2, sizes, 2, seed)
    T_gpu, acc_gpu = swap.temperatures()
    for l, r in enumerate(image):
        T_pred[r] = kT_slot[l] / KB
    np.testing.assert_allclose(T_gpu, T_pred, rtol=1e-13)
    counts = np.zeros(n, np.int32)
    for l in acc1 + acc2:
        counts[l] += 1
    assert np.array_equal(acc_gpu, counts)
    assert len(acc1) + len(acc2) > 0
    # the odd-sized replica keeps its temperature
    assert T_gpu[9] == pytest.approx(T[9], rel=1e-13)


def test_graph_replay_equals_plain_steps_with_swaps():
    import matjes_b200 as mj

    sizes = [(16, 16)] * 6 + [(24, 20)] * 4
    T = list(20.0 + 2.0 * np.arange(len(sizes)))
    cell, B, _ = _square_batch(sizes, np.linspace(0.1, 1.0, len(sizes)), T)
    m0 = mj.random_sphere(sum(a * b for a, b in sizes), 8)
    a = mj.ReplicaBatch(cell, sizes, B, T)
    b = mj.ReplicaBatch(cell, sizes, B, T)
    a.upload(m0)
    b.upload(m0)
    pa = a.params(seed=5, step0=20)
    pb = b.params(seed=5, step0=20)
    a.step(pa, 80, swap_every=10)
    b.graph_run(pb, 20, 4, swap_every=10)
    import torch

    torch.cuda.synchronize()
    assert np.array_equal(a.download(), b.download())
    Ta, acca = a.temperatures()
    Tb, accb = b.temperatures()
    assert np.array_equal(Ta, Tb) and np.array_equal(acca, accb)
    assert pa.step0 == pb.step0 == 100


def test_batch_rejects_what_it_cannot_run():
    import ctypes as C

    import matjes_b200 as mj
    from matjes_b200 import _abi

    cell, B, _ = _square_batch([(8, 8)], [0.0], [1.0])
    batch = mj.ReplicaBatch(cell, [(8, 8)], B, [1.0])
    p = batch.params()
    p.integrator = _abi.MJ_HEUN_MATJES
    assert _abi.lib.mj_batch_step(batch.handle, C.byref(p), 1, 0, None, None) == _abi.MJ_ERR_UNSUPPORTED
    p = batch.params()
    assert _abi.lib.mj_batch_graph_run(batch.handle, C.byref(p), 15, 1, 10, None, None) == _abi.MJ_ERR_ARG
    assert _abi.lib.mj_batch_set_config(batch.handle, 5, 8) == _abi.MJ_ERR_ARG
    dip = mj.square_film((8, 8, 2), a=0.25, med_z=-0.3, dip=True)
    with pytest.raises(mj.MatjesError):
        mj.ReplicaBatch(dip, [(8, 8)], B, [1.0])
    with pytest.raises(mj.MatjesError):
        mj.ReplicaBatch(cell, [(8, 0)], B, [1.0])


def test_full_replica_workload_properties():
    """The 256-replica workload (about 5.1M sites) at full size: unit norm after
    graph replays with swaps, finite energies, the ladder stays a permutation,
    and the smallest replicas still follow their own single-lattice runs."""
    import matjes_b200 as mj

    w = mj.workload("square_replicas256")
    sizes, B, T = w["sizes"], w["B_ext"], w["temperature"]
    batch = mj.ReplicaBatch(w["cell"], sizes, B, T)
    batch.upload(w["m0"])
    d = w["dyn"]
    p = batch.params(timestep=d["timestep"], alpha=d["alpha"], noise="philox", seed=d["seed"])
    batch.graph_run(p, 100, 2, swap_every=d["swap_every"])
    out = batch.download()
    assert np.abs(np.linalg.norm(out, axis=1) - 1.0).max() < 1e-13
    E = batch.energies()
    assert np.all(np.isfinite(E))
    Tn, _ = batch.temperatures()
    np.testing.assert_allclose(np.sort(Tn), np.sort(T), rtol=1e-13)
    # replicas whose temperature never moved: rerun them alone
    small = [r for r in range(len(sizes)) if sizes[r][0] == sizes.min() and abs(Tn[r] - T[r]) <= 1e-12 * T[r]][:3]
    assert small
    for r in small:
        deck = mj.square_film((int(sizes[r][0]), int(sizes[r][1]), 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=B[r, 2])
        m = np.ascontiguousarray(w["m0"][batch.offsets[r]:batch.offsets[r + 1]])
        mj.SpinDynamics(mj.Hamiltonian(deck), integrator="sib", timestep=d["timestep"], alpha=d["alpha"],
                        temperature=T[r], noise="philox", seed=d["seed"], stream_id=r).run(m, 200)
        assert np.abs(batch.replica(out, r) - m).max() <= 1e-13


def test_batch_field_and_energies_of_every_replica():
    """mj_batch_field: each replica's effective field and energy equal its own
    plan's get_eff_field / energy and the oracle's (the GNEB per-image call,
    GNEB/gneb_utils.f90:77-81); the projected field is B - (B.m) m."""
    import matjes_b200 as mj

    cell, B, decks = CASES["square_mixed"]()
    ms = _initial(decks, 31)
    batch = mj.ReplicaBatch(cell, [d.L[:2] for d in decks], B, TEMPS["square_mixed"])
    batch.upload(np.concatenate(ms))
    Bb, Eb = batch.field(project=False)
    Bp, _ = batch.field(project=True, energies=False)
    Bb = Bb.cpu().numpy().T
    Bp = Bp.cpu().numpy().T
    Eb = Eb.cpu().numpy()
    for r, deck in enumerate(decks):
        ref = mj.Hamiltonian(deck).get_eff_field(ms[r])
        got = batch.replica(Bb, r)
        assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max()
        Bo, _ = O.Model(deck).field(ms[r])
        assert np.abs(got - Bo).max() <= 1e-12 * np.abs(Bo).max()
        Eo = O.Model(deck).energy(ms[r])
        assert abs(Eb[r] - Eo) <= E_TOL * abs(Eo)
        proj = got - np.sum(got * ms[r], axis=1, keepdims=True) * ms[r]
        assert np.abs(batch.replica(Bp, r) - proj).max() <= 1e-15 * np.abs(ref).max()


def _tangent_reference(images, E, r, mode):
    """GNEB/tangent.f90: lattice_special (:93-124) or lattice_single (:163-180),
    then vec_project on the image and normalisation over the image."""
    nim = len(images)
    m = images[r]
    if r == 0:
        tau = images[1] - m
    elif r == nim - 1:
        tau = m - images[r - 1]
    elif mode == "central":
        tau = images[r + 1] - images[r - 1]
    else:
        u1, u2, u3 = E[r - 1], E[r], E[r + 1]
        taup, taum = images[r + 1] - m, m - images[r - 1]
        if u3 > u2 > u1:
            tau = taup
        elif u1 > u2 > u3:
            tau = taum
        else:
            dmax, dmin = abs(u3 - u2), abs(u1 - u2)
            if dmax < dmin:
                dmax, dmin = dmin, dmax
            tau = dmax * taup + dmin * taum if u3 > u1 else dmin * taup + dmax * taum
    tau = tau - np.sum(tau * m, axis=1, keepdims=True) * m
    return tau / np.sqrt(np.sum(tau * tau))


@pytest.mark.parametrize("mode", ["energy", "central"])
def test_gneb_tangents_follow_the_reference(mode):
    import matjes_b200 as mj

    nim, L = 7, (24, 20)
    cell, B, decks = _square_batch([L] * nim, [0.3] * nim, [0.0] * nim)
    # a path from +z to a rotated state through random intermediate images
    rng = np.random.default_rng(41)
    n = L[0] * L[1]
    a = np.tile([0.0, 0.0, 1.0], (n, 1))
    b = mj.random_sphere(n, 42)
    images = []
    for k in range(nim):
        t = k / (nim - 1)
        v = (1 - t) * a + t * b + 0.05 * rng.standard_normal((n, 3))
        images.append(v / np.linalg.norm(v, axis=1, keepdims=True))
    batch = mj.ReplicaBatch(cell, [L] * nim, B, [0.0] * nim)
    batch.upload(np.concatenate(images))
    _, E = batch.field()
    tau = batch.gneb_tangent(E, mode=mode).cpu().numpy().T
    Eh = E.cpu().numpy()
    for r in range(nim):
        ref = _tangent_reference(images, Eh, r, mode)
        assert np.abs(batch.replica(tau, r) - ref).max() <= 1e-13, r
