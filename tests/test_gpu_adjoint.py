"""Reverse mode of the SIB trajectory (mj_field_vjp, mj_adjoint_*) on the GPU.

Checked three ways: the field VJP against dense torch float64 matrices built
from the oracle's coupling matrices; the whole backward sweep against torch
autograd through a float64 restatement of the same SIB trajectory (16 x 16
crop, with and without Philox noise); and, at the full 256 x 256 / 500-step /
checkpoint-50 workload, directional derivatives against central finite
differences of the loss (relative step 1e-6).  Gradients must agree within
1e-6 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-6


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _deck(L=(16, 16)):
    import matjes_b200 as mj

    return mj.square_film((L[0], L[1], 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.5)


def test_field_vjp_matches_dense_transpose():
    import torch

    import matjes_b200 as mj
    from tests import sib_torch_reference as R

    deck = mj.square_film((12, 10, 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.7, periodic=(1, 0, 0))
    ham = mj.Hamiltonian(deck)
    rng = np.random.default_rng(4)
    m = mj.random_sphere(deck.nsites, 4)
    v = rng.standard_normal((deck.nsites, 3))
    mt = torch.tensor(m.T.copy(), device="cuda")
    vt = torch.tensor(v.T.copy(), device="cuda")
    gm, gt, gb = mj.field_vjp(ham, mt, vt)
    A = R.unit_matrices(deck)
    terms = mj.deck_terms(deck)
    # B(m) = -sum_t v_t A_t m + zc b: its transpose applied to v, and v . dB/dv_t
    Aall = sum(t * At for t, At in zip(terms, A)).numpy()
    gm_ref = -(Aall @ v.reshape(-1)).reshape(-1, 3)
    assert _rel(gm.cpu().numpy().T, gm_ref) < 1e-13
    gt_ref = [-(v.reshape(-1) @ (At.numpy() @ m.reshape(-1))) for At in A]
    assert _rel(gt.cpu().numpy(), gt_ref) < 1e-13
    assert _rel(gb.cpu().numpy().T, R.zeeman_coefficient(deck) * v) < 1e-15


def test_set_terms_reproduces_fresh_plans():
    import dataclasses

    import torch

    import matjes_b200 as mj

    deck = _deck((20, 18))
    ham = mj.Hamiltonian(deck)
    m = mj.random_sphere(deck.nsites, 5)
    B0 = ham.get_eff_field(m)
    traj = mj.SIBTrajectory(ham, 1)
    traj.set_terms(mj.deck_terms(deck) * 1.0000001)
    traj.set_terms(mj.deck_terms(deck))
    B1 = ham.get_eff_field(m)
    assert np.abs(B1 - B0).max() <= 1e-14 * np.abs(B0).max()
    new = dataclasses.replace(deck, J=[(1, 1, 1, 1.1e-3)], D=[(1, 1, 2, 1, 0.35e-3)], K=[(1, (0.0, 0.0, 1.0), -0.08e-3)])
    traj.set_terms(mj.deck_terms(new))
    B2 = ham.get_eff_field(m)
    B3 = mj.Hamiltonian(new).get_eff_field(m)
    assert np.abs(B2 - B3).max() <= 1e-14 * np.abs(B3).max()
    del torch


def _loss_and_grads_torch(deck, m0, terms, b, target, nsteps, dyn, noise=None):
    import torch

    from tests import sib_torch_reference as R

    A = R.unit_matrices(deck)
    m0t = torch.tensor(m0, requires_grad=True)
    tt = torch.tensor(terms, requires_grad=True)
    bt = torch.tensor(b, requires_grad=True)
    mT = R.trajectory(m0t, tt, bt, A, R.zeeman_coefficient(deck), nsteps, dyn["timestep"], dyn["alpha"], noise)
    loss = ((mT - torch.tensor(target)) ** 2).sum(-1).mean()
    loss.backward()
    return float(loss.detach()), m0t.grad.numpy(), tt.grad.numpy(), bt.grad.numpy(), mT.detach().numpy()


def _gpu_grads(deck, m0, terms, b, target, nsteps, dyn, every, **noise):
    import torch

    import matjes_b200 as mj

    ham = mj.Hamiltonian(deck)
    traj = mj.SIBTrajectory(ham, nsteps, checkpoint_every=every, timestep=dyn["timestep"], alpha=dyn["alpha"], **noise)
    m0t = torch.tensor(m0.T.copy(), device="cuda", requires_grad=True)
    tt = torch.tensor(terms, requires_grad=True)
    bt = torch.tensor(b.T.copy(), device="cuda", requires_grad=True)
    tg = torch.tensor(target.T.copy(), device="cuda")
    mT = traj(m0t, tt, bt)
    loss = ((mT - tg) ** 2).sum(0).mean()
    loss.backward()
    return (float(loss.detach()), m0t.grad.cpu().numpy().T, tt.grad.numpy(), bt.grad.cpu().numpy().T,
            mT.detach().cpu().numpy().T)


def _adj_decks():
    import matjes_b200 as mj

    return {
        "square_16x16": _deck(),                                        # tiled kernels, square NN shape
        "triangular_3_shells": mj.triangular((12, 10), Bz=0.5),         # tiled kernels, three-shell shape
        "cubic_film_open_z": mj.square_film((6, 6, 3), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.5, a=0.25,
                                            med_z=-0.3),                # generic kernels
    }


@pytest.mark.parametrize("name", ["square_16x16", "triangular_3_shells", "cubic_film_open_z"])
def test_adjoint_matches_torch_autograd(name):
    import matjes_b200 as mj

    deck = _adj_decks()[name]
    n = deck.nsites
    rng = np.random.default_rng(6)
    m0 = mj.random_sphere(n, 6)
    target = mj.random_sphere(n, 7)
    b = np.zeros((n, 3))
    b[:, 2] = 0.5 + 0.05 * rng.standard_normal(n)
    terms = mj.deck_terms(deck)
    dyn = dict(timestep=0.1, alpha=0.2)
    ref = _loss_and_grads_torch(deck, m0, terms, b, target, 100, dyn)
    got = _gpu_grads(deck, m0, terms, b, target, 100, dyn, every=30)
    assert _rel(got[4], ref[4]) < 1e-11          # the trajectories themselves
    assert abs(got[0] - ref[0]) <= 1e-11 * abs(ref[0])
    for k, name in ((1, "m0"), (2, "terms"), (3, "bfield")):
        assert _rel(got[k], ref[k]) < GRAD_TOL, name
        assert _rel(got[k], ref[k]) < 1e-9, name  # in practice the two agree to rounding


def test_adjoint_with_philox_noise_matches_torch_autograd():
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi

    deck = _deck((16, 12))
    n = deck.nsites
    m0 = mj.random_sphere(n, 8)
    target = mj.random_sphere(n, 9)
    b = np.tile([0.0, 0.0, 0.5], (n, 1))
    terms = mj.deck_terms(deck)
    dyn = dict(timestep=0.1, alpha=0.2)
    T, seed, stream, nsteps = 30.0, 11, 2, 40
    sigma = np.sqrt(dyn["alpha"] * T * 0.000086173324 * 0.658211928 / dyn["timestep"])
    noise = []
    z = torch.empty((3, n), dtype=torch.float64, device="cuda")
    for k in range(nsteps):
        _abi.check(_abi.lib.mj_philox_normals(seed, k, stream, n, z.data_ptr(), None))
        torch.cuda.synchronize()
        noise.append(torch.tensor(sigma * z.cpu().numpy().T))
    ref = _loss_and_grads_torch(deck, m0, terms, b, target, nsteps, dyn, noise)
    got = _gpu_grads(deck, m0, terms, b, target, nsteps, dyn, every=7, temperature=T, noise="philox", seed=seed,
                     stream_id=stream)
    assert _rel(got[4], ref[4]) < 1e-11
    for k in (1, 2, 3):
        assert _rel(got[k], ref[k]) < GRAD_TOL


def test_checkpoint_spacing_does_not_change_gradients():
    import matjes_b200 as mj

    deck = _deck((40, 24))
    n = deck.nsites
    m0 = mj.random_sphere(n, 12)
    target = mj.random_sphere(n, 13)
    b = np.tile([0.0, 0.0, 0.5], (n, 1))
    terms = mj.deck_terms(deck)
    dyn = dict(timestep=0.1, alpha=0.2)
    res = [_gpu_grads(deck, m0, terms, b, target, 60, dyn, every=e) for e in (1, 7, 60)]
    for r in res[1:]:
        for k in range(5):
            assert np.array_equal(np.asarray(r[k]), np.asarray(res[0][k]))


def test_full_size_gradients_against_finite_differences():
    """256 x 256, 500 SIB steps, checkpoints every 50: loss = mean |m_T - m_target|^2
    with the target from J, D, K = 1.1, 0.35, -0.08 meV and a modulated Bz."""
    import torch

    import matjes_b200 as mj

    w = mj.workload("square256_adjoint")
    deck, d = w["deck"], w["dyn"]
    n = deck.nsites
    ham = mj.Hamiltonian(deck)
    traj = mj.SIBTrajectory(ham, d["steps"], checkpoint_every=d["checkpoint_every"], timestep=d["timestep"],
                            alpha=d["alpha"])
    dev = "cuda"
    m0 = torch.tensor(w["m0"].T.copy(), device=dev)
    b = torch.tensor(w["bfield"].T.copy(), device=dev)
    terms = mj.deck_terms(deck)
    # the target trajectory
    traj.set_terms(w["target_terms"])
    traj.set_bfield(torch.tensor(w["target_bfield"].T.copy(), device=dev))
    target = traj.forward(m0).clone()

    def loss(m0_, terms_, b_):
        traj.set_terms(terms_)
        traj.set_bfield(b_)
        mT = traj.forward(m0_)
        return float(((mT - target) ** 2).sum(0).mean())

    m0g = m0.clone().requires_grad_(True)
    tg = torch.tensor(terms, requires_grad=True)
    bg = b.clone().requires_grad_(True)
    mT = traj(m0g, tg, bg)
    L = ((mT - target) ** 2).sum(0).mean()
    L.backward()
    g_m0, g_t, g_b = m0g.grad, tg.grad.numpy(), bg.grad
    rng = np.random.default_rng(14)
    # coupling terms, relative step 1e-6
    for t in range(len(terms)):
        h = 1e-6 * abs(terms[t])
        tp, tm = terms.copy(), terms.copy()
        tp[t] += h
        tm[t] -= h
        fd = (loss(m0, tp, b) - loss(m0, tm, b)) / (2 * h)
        assert abs(fd - g_t[t]) <= GRAD_TOL * abs(g_t[t]), (t, fd, g_t[t])
    # initial spins and per-site field along random directions
    for g, which in ((g_m0, "m0"), (g_b, "b")):
        delta = torch.tensor(rng.standard_normal((3, n)), device=dev)
        h = 1e-6
        if which == "m0":
            fd = (loss(m0 + h * delta, terms, b) - loss(m0 - h * delta, terms, b)) / (2 * h)
        else:
            fd = (loss(m0, terms, b + h * delta) - loss(m0, terms, b - h * delta)) / (2 * h)
        ad = float((g * delta).sum())
        assert abs(fd - ad) <= GRAD_TOL * abs(ad), (which, fd, ad)


@pytest.mark.parametrize("thermal", [False, True])
def test_adjoint_forward_is_the_plain_forward(thermal):
    """The adjoint's forward sweep runs the plan's own SIB kernels: its m_T is
    the state mj_step_dev reaches, bit for bit."""
    import torch

    import matjes_b200 as mj

    deck = _deck((64, 48))
    ham = mj.Hamiltonian(deck)
    noise = dict(temperature=20.0, noise="philox", seed=3, stream_id=1) if thermal else {}
    traj = mj.SIBTrajectory(ham, 40, checkpoint_every=9, timestep=0.1, alpha=0.2, **noise)
    m0 = torch.tensor(mj.random_sphere(deck.nsites, 15).T.copy(), device="cuda")
    mT = traj.forward(m0)
    m = m0.clone()
    mj.SpinDynamics(ham, integrator="sib", timestep=0.1, alpha=0.2, **noise).run(m, 40)
    torch.cuda.synchronize()
    assert torch.equal(mT, m)
