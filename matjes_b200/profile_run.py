"""Run a few LLG steps of a synthetic workload, for profilers (ncu) to capture.

    python -m matjes_b200.profile_run --lattice triangular --L 4096 --T 10 \
        --integrator sib --variant 2 --steps 3

--variant: -1 generic kernel, 0..3 tiled tile shapes, "auto" = the autotuner's pick.

    python -m matjes_b200.profile_run --adjoint --L 256 --steps 20 --every 10

runs one forward + backward sweep of the reverse-mode SIB trajectory instead;

    python -m matjes_b200.profile_run --batch --steps 3

steps the 256-replica batch workload;

    python -m matjes_b200.profile_run --mc --lattice square --L 2048 --steps 3

runs Metropolis sweeps (cone proposals, 10 K) instead of time steps;

    python -m matjes_b200.profile_run --gneb --L 256 --nim 16 --steps 64

relaxes a GNEB path of --nim images of an L x L DMI film (J + D + K + Bz =
0.3 T, periodic; geodesic from +z to -z, interior spins moved by up to 1e-2)
for --steps iterations (force tolerance 0); with --plan the images are held on
the deck's plan (mj_gneb_path) instead of as the replicas of a batch.
"""
from __future__ import annotations

import argparse

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--lattice", default="triangular", choices=["triangular", "square", "film"])
    ap.add_argument("--L", type=int, default=4096)
    ap.add_argument("--Lz", type=int, default=16)
    ap.add_argument("--T", type=float, default=10.0)
    ap.add_argument("--integrator", default="sib")
    ap.add_argument("--variant", default="auto")
    ap.add_argument("--tma", type=int, default=1, help="halo staging of the tiled kernels: 1 TMA, 0 plain loads")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--adjoint", action="store_true", help="one forward + backward sweep of the SIB adjoint")
    ap.add_argument("--every", type=int, default=50, help="adjoint checkpoint spacing")
    ap.add_argument("--batch", action="store_true", help="step the 256-replica batch workload")
    ap.add_argument("--mc", action="store_true", help="Metropolis sweeps (cone proposals) instead of time steps")
    ap.add_argument("--gneb", action="store_true", help="GNEB path relaxation iterations instead of time steps")
    ap.add_argument("--nim", type=int, default=16, help="GNEB images")
    ap.add_argument("--plan", action="store_true", help="GNEB images held on the deck's plan (mj_gneb_path)")
    a = ap.parse_args(argv)
    if a.gneb:
        return gneb(a)
    if a.adjoint:
        return adjoint(a)
    if a.batch:
        return batch(a)

    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi

    if a.lattice == "triangular":
        deck = mj.triangular((a.L, a.L))
        m0 = mj.reversed_disks(deck, 20, 8.0, 1)
    elif a.lattice == "square":
        deck = mj.square_film((a.L, a.L, 1))
        m0 = mj.random_sphere(deck.nsites, 0)
    else:
        deck = mj.square_film((a.L, a.L, a.Lz), Jv=1e-3, Dv=0.15e-3, Kv=-0.02e-3, Bz=0.2, a=0.25, med_z=-0.3, dip=True)
        m0 = mj.random_sphere(deck.nsites, 4)
    ham = mj.Hamiltonian(deck)
    m = torch.tensor(m0.T.copy(), device="cuda")
    if a.mc:
        from matjes_b200.montecarlo import MetropolisMC

        ch = MetropolisMC(ham, "sphere", cone=0.5, seed=3, adapt_cone=False)
        E, _, acc = ch.sweeps(m, a.steps, a.T)
        torch.cuda.synchronize()
        print("ok", ch.colors, acc, E.tolist())
        return
    sd = mj.SpinDynamics(ham, integrator=a.integrator, timestep=0.1, alpha=0.1, temperature=a.T, noise="philox", seed=1)
    sd.p.energy_mode = _abi.MJ_ENERGY_BEFORE
    if a.variant == "auto":
        best = _abi.C.c_int32()
        _abi.check(_abi.lib.mj_plan_autotune(ham.plan, m.data_ptr(), _abi.C.byref(sd.p), 3, _abi.C.byref(best), None,
                                             None))
    elif ham.noffsets:
        _abi.check(_abi.lib.mj_plan_set_variant(ham.plan, int(a.variant)))
        _abi.check(_abi.lib.mj_plan_set_tma(ham.plan, int(a.tma)))
    E = torch.zeros(a.steps + 1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for k in range(a.steps):
        sd.p.step0 = k
        _abi.check(_abi.lib.mj_step_dev(ham.plan, m.data_ptr(), _abi.C.byref(sd.p), 1, E[k:].data_ptr(), stream))
    torch.cuda.synchronize()
    print("ok", E[: a.steps].tolist())


def adjoint(a):
    import torch

    import matjes_b200 as mj

    deck = mj.square_film((a.L, a.L, 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.5)
    ham = mj.Hamiltonian(deck)
    traj = mj.SIBTrajectory(ham, a.steps, checkpoint_every=a.every, timestep=0.1, alpha=0.2)
    rng = np.random.default_rng(3)
    b = torch.tensor(np.stack([np.zeros(deck.nsites), np.zeros(deck.nsites),
                               0.5 + 0.05 * rng.standard_normal(deck.nsites)]), device="cuda")
    traj.set_bfield(b)
    m0 = torch.tensor(mj.random_sphere(deck.nsites, 3).T.copy(), device="cuda")
    mT = traj.forward(m0)
    g0, gt, gb = traj.backward(mT - m0)
    torch.cuda.synchronize()
    print("ok", gt.tolist(), float(g0.abs().sum()), float(gb.abs().sum()))


def gneb(a):
    import matjes_b200 as mj
    from matjes_b200.gneb import geodesic_path

    deck = mj.square_film((a.L, a.L, 1), Jv=1e-3, Dv=0.4e-3, Kv=-0.2e-3, Bz=0.3, mu_s=2.0, periodic=(1, 1, 0))
    n = a.L * a.L
    up = np.tile([0.0, 0.0, 1.0], (n, 1))
    path = geodesic_path(up, -up, a.nim, amp_rnd=1e-2, seed=1)
    path[0], path[-1] = up, -up
    if a.plan:
        from matjes_b200.gneb import PlanPath

        bt = PlanPath(mj.Hamiltonian(deck), path)
    else:
        bt = mj.ReplicaBatch(deck, [(a.L, a.L)] * a.nim, np.tile(deck.B_ext, (a.nim, 1)), [0.0] * a.nim)
        bt.upload(path.reshape(-1, 3))
    rx, ene, dene, its, fchk, _ = bt.gneb_path(0.3, 0.02, 1.0, 0.0, a.steps, "I")
    print("ok", its, fchk, ene.tolist())


def batch(a):
    import torch

    import matjes_b200 as mj

    w = mj.workload("square_replicas256")
    bt = mj.ReplicaBatch(w["cell"], w["sizes"], w["B_ext"], w["temperature"])
    bt.upload(w["m0"])
    d = w["dyn"]
    p = bt.params(timestep=d["timestep"], alpha=d["alpha"], noise="philox", seed=d["seed"])
    bt.step(p, a.steps)
    torch.cuda.synchronize()
    print("ok", bt.energies()[:4].tolist())


if __name__ == "__main__":
    main()
