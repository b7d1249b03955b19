"""Run a few LLG steps of a synthetic workload, for profilers (ncu) to capture.

    python -m matjes_b200.profile_run --lattice triangular --L 4096 --T 10 \
        --integrator sib --variant 2 --steps 3

--variant: -1 generic kernel, 0..3 tiled tile shapes, "auto" = the autotuner's pick.
"""
from __future__ import annotations

import argparse


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
    a = ap.parse_args(argv)

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


if __name__ == "__main__":
    main()
