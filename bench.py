#!/usr/bin/env python
"""Throughput of the Matjes LLG hot path on B200: spin-updates/s and HBM roofline.

Workload (default): the 1024x1024 periodic triangular monolayer with exchange
shells J1..J3 = 1.0, -0.1, -0.05 meV, interfacial D1 = 0.2 meV, K = 0.05 meV
easy axis, Bz = 1 T, SIB integrator, alpha = 0.1, dt = 0.1 fs, T = 10 K with
Philox thermal noise (seed 1), initial state: +z ferromagnet with 20 reversed
disks of radius 8.  One bench step = one full LLG time step over the lattice
(both SIB passes, with the total energy of the incoming state fused into the
first pass).  Synthetic data of the stated shapes; nothing is read from disk.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs one process per GPU (torchrun); the path does not shard, so every
rank runs its own replica (Philox stream = rank) and the value is the sum over
ranks with the time the max over ranks ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

UNIT = "spin-updates/s"
FLUSH_BYTES = 256 << 20  # larger than the 126 MB L2


# the benchmark's metric, as the reference's headline figure names it
METRIC = "LLG spin-updates/s & HBM GB/s at 1e-12 field err; batched/adjoint vs plain, 1 B200"


def metric_name() -> str:
    return METRIC


def peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "source": "fallback"}


# both arms compute, per step, the energy of the state the step starts from
ENERGY_CONVENTION = "energy of the incoming state, fused into the first field pass"


def workload_config(name, deck, dyn, extra=None) -> dict:
    cfg = {
        "workload": name,
        "lattice": f"{deck.L[0]}x{deck.L[1]}x{deck.L[2]} triangular, periodic in-plane" if "triangular" in name
        else f"{deck.L[0]}x{deck.L[1]}x{deck.L[2]}",
        "terms": "J1,J2,J3 + D1 (hollow-site mediators) + uniaxial K + Zeeman",
        "integrator": dyn["integrator"],
        "timestep_fs": dyn["timestep"],
        "alpha": dyn["alpha"],
        "temperature_K": dyn["temperature"],
        "noise": dyn.get("noise", "off"),
        "sites": int(deck.nsites),
        "l2": "flushed before every timed step: 256 MiB written, then 256 MiB of another buffer read",
    }
    if extra:
        cfg.update(extra)
    return cfg


# ----------------------------------------------------------------------
class Clocks:
    """SM clock and clock-event (throttle) reasons polled through NVML every
    0.5 ms while the timed region runs (read-only queries)."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, cuda_index: int):
        self.samples, self.reasons, self.err = [], set(), None
        self.handle = None
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            pr = torch.cuda.get_device_properties(cuda_index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
        except Exception as e:  # noqa: BLE001
            self.err = f"nvml unavailable: {e}"

    def _poll(self):
        nv = self.nvml
        while not self._stop:
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)))
                r = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle))
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception as e:  # noqa: BLE001
                self.err = str(e)
                return
            time.sleep(0.0005)

    def start(self):
        import threading

        if self.handle is None:
            return
        self._stop = False
        self.th = threading.Thread(target=self._poll, daemon=True)
        self.th.start()

    def stop(self) -> dict:
        if self.handle is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.err or "no nvml"]}
        self._stop = True
        self.th.join()
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [self.err or "no samples"]}
        return {"sm_mhz": float(np.median(self.samples)), "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples), "source": "nvml"}


def ncu_figure(name: str, kernel: str, summary: str = "k_tiled_sib_triangular2048.md"):
    """A per-kernel figure (`<name> <kernel>: value`) of the committed ncu summary
    of the SIB passes on a 2048^2 lattice; None if there is none."""
    fn = os.path.join(ROOT, "profiles", summary)
    if not os.path.exists(fn):
        return None
    m = re.search(r"%s %s:\s*([0-9.eE+-]+)" % (re.escape(name), re.escape(kernel)), open(fn).read())
    return float(m.group(1)) if m else None


def ncu_traffic(kernel: str):
    """DRAM bytes (read + write) per site of one launch of `kernel` (the passes
    stream their fields once, so the traffic scales with the site count)."""
    return ncu_figure("dram_bytes_per_site", kernel)


# ----------------------------------------------------------------------
# replicas-only multi-GPU: every rank advances its own replica of the workload
def replica_stream(rank: int) -> int:
    """Philox stream of a rank's replica: replicas draw independent noise."""
    return int(rank)


def max_over_ranks(x: float, device, dist: bool) -> float:
    """The maximum of a per-rank figure (the job's time is its slowest rank's)."""
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist:
        import torch.distributed as td

        td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def job_rate(sites: int, steps: int, world: int, seconds: float) -> float:
    """Whole-job spin-updates/s: every rank advanced `sites` x `steps`."""
    return sites * steps * world / seconds


# ----------------------------------------------------------------------
def cpu_oracle_rate(wname, seconds=15.0):
    """The oracle (C restatement, -O3 -march=native, OpenMP over all host
    threads) on a bounded sample of the same workload: the full lattice, the
    same couplings and dynamics, as many steps as fit in about `seconds`, with
    the energy of each step's incoming state fused as in the GPU arm; then the
    same on one core."""
    workload = deck_module().workload
    O = oracle_native()

    w = workload(wname)
    dyn = dict(w["dyn"])
    dyn.pop("steps")
    M = O.Model(w["deck"])
    m = w["m0"].copy()
    N = w["deck"].nsites
    t = time.perf_counter()
    M.run(m, 2, energies=True, energy_before=True, **dyn)
    per = (time.perf_counter() - t) / 2
    nst = int(max(3, min(2000, seconds / max(per, 1e-6))))
    t = time.perf_counter()
    M.run(m, nst, step0=2, energies=True, energy_before=True, **dyn)
    el = time.perf_counter() - t
    # the same on one core (a few seconds)
    O.set_threads(1)
    n1 = max(1, int(min(nst, 0.3 * seconds / max(per * (os.cpu_count() or 1), 1e-6))))
    t = time.perf_counter()
    M.run(m, n1, step0=2 + nst, energies=True, energy_before=True, **dyn)
    el1 = time.perf_counter() - t
    O.set_threads(0)
    L = w["deck"].L
    return {"value": N * nst / el, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"oracle SIB+Philox, full {L[0]}x{L[1]} lattice, {nst} steps, {el:.1f} s, "
                      f"energy of the incoming state fused",
            "build": "oracle/liboracle_native.so (-O3 -march=native -fopenmp -ffp-contract=off, built on this host)",
            "single_core": {"value": N * n1 / el1, "unit": UNIT, "cores": 1,
                            "sample": f"the same, {n1} steps, {el1:.1f} s"}}


def deck_module():
    """matjes_b200/deck.py loaded by its path, outside the package: the package's
    import loads the CUDA library, which the CPU legs have no use for."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("matjes_deck_cpu", os.path.join(ROOT, "matjes_b200", "deck.py"))
    if spec.name in sys.modules:
        return sys.modules[spec.name]
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # dataclasses look their module up while the file runs
    spec.loader.exec_module(mod)
    return mod


def oracle_native():
    """The oracle built -O3 -march=native on this machine (the CPU legs' timed
    build; the tests use the portable -O2 build of the same source)."""
    os.environ["ORACLE_NATIVE"] = "1"
    from oracle import oracle as O

    return O


def run_reference(args, rank, world):
    """--impl reference: the oracle port (the reference cannot be compiled here:
    no Fortran compiler) on the full workload, all host threads, with the
    energy of the state each step starts from summed in its first field pass,
    the convention of the GPU arm."""
    if rank != 0:
        return
    workload = deck_module().workload
    O = oracle_native()

    w = workload(args.workload)
    dyn = dict(w["dyn"])
    dyn.pop("steps")
    M = O.Model(w["deck"])
    m = w["m0"].copy()
    M.run(m, args.warmup, **dyn)
    t = time.perf_counter()
    E = M.run(m, args.steps, step0=args.warmup, energies=True, energy_before=True, **dyn)
    el = time.perf_counter() - t
    N = w["deck"].nsites
    value = N * args.steps / el
    line = {
        "metric": metric_name(), "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": workload_config(args.workload, w["deck"], w["dyn"],
                                  {"parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "single",
                                   "energy_per_step": ENERGY_CONVENTION}),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                         "sample": f"full {w['deck'].L[0]}x{w['deck'].L[1]} lattice, {args.steps} SIB steps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "final_energy_eV": float(E[-1]),
        "oracle_build": "oracle/liboracle_native.so: -O3 -march=native -fopenmp -ffp-contract=off, built on this host",
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------
def run_batch(dev: int, steps: int = 200) -> dict:
    """The 256-replica workload (square lattices of sides 32..256, about 5.1M
    sites, Bz ~ U(0,2) T, T geometric 1..50 K, SIB alpha = 0.5, Philox, a
    parallel-tempering round every 100 steps): one batch advanced by CUDA
    graphs of 100 steps against the same replicas run one after another
    through their own plans (mj_step_dev, and mj_graph_run of 100 steps)."""
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi
    from matjes_b200.deck import square_film, workload

    w = workload("square_replicas256")
    d = w["dyn"]
    sizes, B, T = w["sizes"], w["B_ext"], w["temperature"]
    spg = int(d["swap_every"])
    nrg = max(1, steps // spg)
    steps = spg * nrg
    b = mj.ReplicaBatch(w["cell"], sizes, B, T, device=dev)
    b.upload(w["m0"])
    N = b.N
    p = b.params(timestep=d["timestep"], alpha=d["alpha"], noise="philox", seed=d["seed"])
    (v, bps), table = b.autotune(p, steps=5)
    b.graph_run(p, spg, 1, swap_every=spg)  # capture + one warm replay
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.graph_run(p, spg, nrg, swap_every=spg)
    e1.record()
    torch.cuda.synchronize()
    ms_batch = e0.elapsed_time(e1)
    Tn, acc = b.temperatures()
    b.close()

    # the same replicas, one plan each, run one after another
    plans = []
    for r in range(len(sizes)):
        deck = square_film((int(sizes[r][0]), int(sizes[r][1]), 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=B[r, 2])
        ham = mj.Hamiltonian(deck, device=dev)
        sd = mj.SpinDynamics(ham, integrator="sib", timestep=d["timestep"], alpha=d["alpha"], temperature=T[r],
                             noise="philox", seed=d["seed"], stream_id=r)
        m = torch.tensor(w["m0"][int(np.sum(sizes[:r, 0].astype(np.int64) * sizes[:r, 1]))
                                 :int(np.sum(sizes[:r + 1, 0].astype(np.int64) * sizes[:r + 1, 1]))].T.copy(),
                         device=f"cuda:{dev}")
        st = mj.SpinState(ham)
        st.device_tensor().copy_(m)
        plans.append((ham, sd, m, st))
    lib = _abi.lib

    def sequential(nsteps, graphs):
        for ham, sd, m, st in plans:
            if graphs:
                _abi.check(lib.mj_graph_run(ham.plan, st.handle, _abi.C.byref(sd.p), spg, nsteps // spg, None, None))
            else:
                _abi.check(lib.mj_step_dev(ham.plan, m.data_ptr(), _abi.C.byref(sd.p), nsteps, None, None))
            sd.p.step0 += nsteps

    res = {}
    for graphs in (False, True):
        sequential(spg, graphs)  # warm-up (and graph capture)
        torch.cuda.synchronize()
        e0.record()
        sequential(steps, graphs)
        e1.record()
        torch.cuda.synchronize()
        res[graphs] = e0.elapsed_time(e1)
    su_batch = N * steps / (ms_batch / 1e3)
    return {
        "workload": "square_replicas256", "replicas": int(len(sizes)), "sites": int(N), "steps": steps,
        "swap_every": spg, "tile_variant": int(v), "blocks_per_sm": int(bps),
        "value": su_batch, "unit": UNIT, "ms_per_step": ms_batch / steps,
        "achieved_gbs": 120.0 * N * steps / (ms_batch / 1e3) / 1e9,
        "sequential_plain": {"value": N * steps / (res[False] / 1e3), "ms_per_step": res[False] / steps,
                             "path": "256 plans, mj_step_dev one replica after another"},
        "sequential_graphs": {"value": N * steps / (res[True] / 1e3), "ms_per_step": res[True] / steps,
                              "path": "256 plans, mj_graph_run (100-step graphs) one replica after another"},
        "speedup_vs_sequential_plain": res[False] / ms_batch,
        "speedup_vs_sequential_graphs": res[True] / ms_batch,
        "swaps_accepted": int(acc.sum()),
        "autotune_ms_per_step": np.round(table, 5).tolist(),
    }


def run_adjoint(dev: int, reps: int = 3) -> dict:
    """The 256 x 256 adjoint workload (square lattice, J, D, K + per-site Bz,
    SIB alpha = 0.2, 500 steps, checkpoints every 50): one forward + backward
    sweep (gradients for m0, the three coupling terms and the per-site field)
    against the plain 500-step forward through mj_step_dev."""
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi
    from matjes_b200.deck import workload

    w = workload("square256_adjoint")
    deck, d = w["deck"], w["dyn"]
    N = deck.nsites
    ham = mj.Hamiltonian(deck, device=dev)
    b = torch.tensor(w["bfield"].T.copy(), device=f"cuda:{dev}")
    m0 = torch.tensor(w["m0"].T.copy(), device=f"cuda:{dev}")
    target = torch.tensor(mj.random_sphere(N, 7).T.copy(), device=f"cuda:{dev}")
    traj = mj.SIBTrajectory(ham, d["steps"], checkpoint_every=d["checkpoint_every"], timestep=d["timestep"],
                            alpha=d["alpha"])
    traj.set_bfield(b)
    sd = mj.SpinDynamics(ham, integrator="sib", timestep=d["timestep"], alpha=d["alpha"])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def plain():
        m = m0.clone()
        sd.run(m, d["steps"], step0=0)
        return m

    st = mj.SpinState(ham)

    def plain_graph():
        st.device_tensor().copy_(m0)
        sd.p.step0 = 0
        _abi.check(_abi.lib.mj_graph_run(ham.plan, st.handle, _abi.C.byref(sd.p), d["steps"], 1, None, None))

    def adjoint():
        mT = traj.forward(m0)
        g = 2.0 * (mT - target) / N
        return traj.backward(g)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(reps):
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    f = timed(plain)
    fg = timed(plain_graph)
    a = timed(adjoint)
    return {"workload": "square256_adjoint", "sites": N, "steps": d["steps"],
            "checkpoint_every": d["checkpoint_every"], "forward_ms": f, "forward_graph_ms": fg,
            "forward_backward_ms": a, "cost_ratio": a / f, "cost_ratio_vs_graph_forward": a / fg,
            "gradients": "m0 (3N), J, D, K, per-site B (3N)",
            "launches_per_step": {"forward": 2, "adjoint": 6},
            "adjoint_path": "forward and backward sweeps replayed as CUDA graphs"}


def dipolar_alg_bytes(N: int, nrep) -> float:
    """Compulsory bytes of one FFT dipolar evaluation (FP64, 3 components): pad
    (read 24 N, write 24 Np), D2Z (read 24 Np, write 48 Nc), pointwise (read the
    symmetric complex K_F 96 Nc and M_F 48 Nc, write 48 Nc), Z2D (read 48 Nc,
    write 24 Np), unpack (read H 24 N, read and write B 48 N); Np = prod(N_rep),
    Nc = Np / N_rep,x * (N_rep,x / 2 + 1).  About 140 MB on the 128 x 128 x 32
    grid of the 128 x 128 x 16 film."""
    Np = int(np.prod(nrep))
    Nc = Np // nrep[0] * (nrep[0] // 2 + 1)
    return 24.0 * N + 24.0 * Np + 24.0 * Np + 48.0 * Nc + 96.0 * Nc + 48.0 * Nc + 48.0 * Nc + 48.0 * Nc + \
        24.0 * Np + 24.0 * N + 48.0 * N


def run_dipolar(dev: int, steps: int = 50) -> dict:
    """The dipolar film (128 x 128 x 16 simple cubic, a = 0.25 nm, periodic in-plane,
    open along z, J + D + K + Zeeman + FFT dipolar, SIB alpha = 0.1, T = 5 K
    Philox) on the reference's grid (128 x 128 x 32) and on the fully zero-padded
    one (256 x 256 x 32, every axis padded to twice the lattice): one system
    each, and on the reference's grid 8 systems with their own initial states
    (seeds 4..11) advanced concurrently on 8 CUDA streams.  Each grid's dipolar
    evaluation (pad, transforms, pointwise product; the unpack is fused into the
    passes) gets its roofline against dipolar_alg_bytes."""
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi
    from matjes_b200.deck import workload

    lib = _abi.lib
    pk = peaks()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def make(dip, k):
        w = workload("film128x16_dipolar")
        deck, d = w["deck"], dict(w["dyn"])
        d.pop("steps")
        deck.dip = dip
        ham = mj.Hamiltonian(deck, device=dev)
        sd = mj.SpinDynamics(ham, stream_id=k, **d)
        m = torch.tensor(mj.random_sphere(deck.nsites, 4 + k).T.copy(), device=f"cuda:{dev}")
        return ham, sd, m, torch.cuda.Stream(device=dev)

    def run(sys_list, nsteps, concurrent):
        for ham, sd, m, st in sys_list:
            s = st.cuda_stream if concurrent else torch.cuda.current_stream().cuda_stream
            _abi.check(lib.mj_step_dev(ham.plan, m.data_ptr(), _abi.C.byref(sd.p), nsteps, None, s))
            sd.p.step0 += nsteps

    def timed(sys_list, concurrent):
        run(sys_list, 3, concurrent)
        torch.cuda.synchronize()
        e0.record()
        for _, _, _, st in sys_list:
            st.wait_event(e0)
        run(sys_list, steps, concurrent)
        for _, _, _, st in sys_list:
            torch.cuda.current_stream().wait_stream(st)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    out = {"workload": "film128x16_dipolar", "steps": steps}
    for dip, key in ((1, "reference_grid"), (2, "padded_grid")):
        one = make(dip, 0)
        ham = one[0]
        N = ham.N
        t = timed([one], False)
        _abi.check(lib.mj_profile_enable(ham.plan, 1))
        run([one], 5, False)
        prof = _abi.profile_read(ham.plan)
        _abi.check(lib.mj_profile_enable(ham.plan, 0))
        tot = sum(v for v, _ in prof.values())
        nrep = (128, 128, 32) if dip == 1 else (256, 256, 32)
        d_ms, d_n = prof.get("dipolar_fft", (0.0, 1))
        per_eval = d_ms / max(d_n, 1)
        b = dipolar_alg_bytes(N, nrep)
        out[key] = {"fft_grid": list(nrep), "sites": N, "value": N * steps / (t / 1e3), "unit": UNIT,
                    "ms_per_step": t / steps, "kernel_share": {k: round(v / tot, 4) for k, (v, _) in prof.items()},
                    "dipolar_eval": {"us": 1e3 * per_eval, "alg_bytes": b, "achieved_gbs": b / (per_eval / 1e3) / 1e9,
                                     "frac": b / (per_eval / 1e3) / 1e9 / pk["hbm_gbs"], "peak_source": pk["source"]}}
        if dip == 1:
            systems = [one] + [make(1, k) for k in range(1, 8)]
            eight = timed(systems, True)
            out[key]["batch8"] = {"value": 8 * N * steps / (eight / 1e3), "ms_per_step": eight / steps,
                                  "path": "8 plans, mj_step_dev on 8 CUDA streams"}
            del systems
        del one
    out["value"] = out["reference_grid"]["value"]
    return out


def run_hbm_resident(dev: int, steps: int = 20) -> dict:
    """The bench workload at 4096^2 (triangular1024_thermal's couplings and
    dynamics, 16.8 M sites, 403 MB per field, so every pass streams from HBM with
    no L2 flush needed): the variant autotuned by the library on this lattice,
    then `steps` timed SIB steps, with the per-kernel roofline of the two passes."""
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi
    from matjes_b200.deck import workload

    w = workload("triangular4096_thermal")
    deck, dyn = w["deck"], dict(w["dyn"])
    dyn.pop("steps")
    N = deck.nsites
    ham = mj.Hamiltonian(deck, device=dev)
    sd = mj.SpinDynamics(ham, **dyn)
    p = sd.p
    p.energy_mode = _abi.MJ_ENERGY_BEFORE
    m = torch.tensor(w["m0"].T.copy(), device=f"cuda:{dev}")
    lib = _abi.lib
    best, best_tma = _abi.C.c_int32(), _abi.C.c_int32()
    _abi.check(lib.mj_plan_autotune(ham.plan, m.data_ptr(), _abi.C.byref(p), 3, _abi.C.byref(best),
                                    _abi.C.byref(best_tma), None))
    E = torch.zeros(steps + 64, dtype=torch.float64, device=m.device)
    stream = torch.cuda.current_stream().cuda_stream
    # the fields (403 MB each) exceed L2: no flush between the tuning steps
    cfg, _ = tune_kernels(lib, _abi, ham.plan, m, p, lambda: None, E, stream, variants=False)
    cfg.update(variant=int(best.value), tma=int(best_tma.value))
    for k in range(3):
        p.step0 = k
        _abi.check(lib.mj_step_dev(ham.plan, m.data_ptr(), _abi.C.byref(p), 1, E.data_ptr(), stream))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    p.step0 = 3
    _abi.check(lib.mj_step_dev(ham.plan, m.data_ptr(), _abi.C.byref(p), steps, E.data_ptr(), stream))
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    _abi.check(lib.mj_profile_enable(ham.plan, 1))
    p.step0 = 100
    _abi.check(lib.mj_step_dev(ham.plan, m.data_ptr(), _abi.C.byref(p), 5, E.data_ptr(), stream))
    prof = _abi.profile_read(ham.plan)
    _abi.check(lib.mj_profile_enable(ham.plan, 0))
    pk = peaks()
    kern = {}
    for name, b in (("k_sib1", 48.0), ("k_sib2", 72.0), ("k_sib_fused", 120.0)):
        if name in prof:
            tot, cnt = prof[name]
            avg = tot / max(cnt, 1)
            gbs = b * N / (avg / 1e3) / 1e9
            kern[name] = {"avg_us": 1e3 * avg, "achieved_gbs": gbs, "frac": gbs / pk["hbm_gbs"]}
    return {"workload": "triangular4096_thermal", "sites": N, "steps": steps, "kernels_config": cfg,
            "value": N / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
            "step_roofline": {"alg_bytes_per_site": 120.0, "achieved_gbs": 120.0 * N / (ms / 1e3) / 1e9,
                              "frac": 120.0 * N / (ms / 1e3) / 1e9 / pk["hbm_gbs"]},
            "kernels": kern}


def run_monte_carlo(dev: int, sweeps: int = 100) -> dict:
    """Metropolis Monte Carlo: the square film 1024 x 1024 (J + D + K + Bz = 0.5 T,
    cone proposals, 10 K, 2-colour checkerboard sweeps) on one chain; 256 replicas
    of 64 x 64 (temperatures geometric 1..50 K) with a parallel-tempering round
    every 10 sweeps; and, as the CPU baseline, the oracle's random-site chain on one
    host core (256 x 256, the reference's move order).  Consecutive sweeps keep the 25 MB spin field in
    L2, as a chain does; the rates are moves per second."""
    import time

    import numpy as np
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi
    from matjes_b200.montecarlo import MetropolisMC
    from oracle import oracle as O

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    deck = mj.square_film((1024, 1024, 1))
    ham = mj.Hamiltonian(deck, device=dev)
    m = torch.tensor(mj.random_sphere(deck.nsites, 1).T.copy(), device=f"cuda:{dev}")
    ch = MetropolisMC(ham, "sphere", cone=0.5, seed=3, adapt_cone=False)
    ch.sweeps(m, 5, 10.0, record=False)
    torch.cuda.synchronize()
    e0.record()
    ch.sweeps(m, sweeps, 10.0, record=False)
    e1.record()
    torch.cuda.synchronize()
    one = e0.elapsed_time(e1)
    n = 256
    batch = mj.ReplicaBatch(mj.square_film((8, 8, 1)), [(64, 64)] * n, np.zeros((n, 3)),
                            list(np.geomspace(1.0, 50.0, n)), device=dev)
    batch.upload(mj.random_sphere(64 * 64 * n, 2))
    p = _abi.McParams(0.0, 0.5, _abi.MJ_MC_CONE, 1, 5, 0, 0, 0, 0, 0, 0)
    batch.monte_carlo(p, 2, 10, swap=True, record=False)
    torch.cuda.synchronize()
    e0.record()
    batch.monte_carlo(p, sweeps // 10, 10, swap=True, record=False)
    e1.record()
    torch.cuda.synchronize()
    bt = e0.elapsed_time(e1)
    cdeck = mj.square_film((256, 256, 1))
    mo = mj.random_sphere(cdeck.nsites, 1)
    st = O.MC(temperature=10.0, cone=0.5, proposal=0, adapt_cone=0, seed=3, stream_id=0, sweep0=0)
    model = O.Model(cdeck)
    t0 = time.perf_counter()
    O.mc_random(model, mo, st, 60)
    ct = time.perf_counter() - t0
    return {"workload": "square1024_mc", "sites": deck.nsites, "sweeps": sweeps, "colours": list(ch.colors),
            "value": deck.nsites * sweeps / (one / 1e3), "unit": "moves/s", "us_per_sweep": 1e3 * one / sweeps,
            "acceptance": ch.rate,
            "batch": {"workload": "square64_replicas256_ptmc", "sites": batch.N, "swap_every": 10,
                      "value": batch.N * sweeps / (bt / 1e3), "unit": "moves/s", "us_per_sweep": 1e3 * bt / sweeps},
            "cpu_baseline": {"value": cdeck.nsites * 60 / ct, "unit": "moves/s", "cores": 1, "kind": "port",
                             "sample": "256x256 square film, 60 sweeps of random-site moves (orc_mc_random)"}}


def run_gneb(dev: int, nim: int = 16, side: int = 256) -> dict:
    """GNEB path relaxation (find_path, velocity projection): a DMI film side x
    side (J + D + K + Bz = 0.3 T, periodic) with a path of nim images from +z to
    -z (geodesic, every interior spin moved by up to 1e-2), max |F| tolerance 0
    so that every call runs its itrmax iterations.  The iteration rate is the
    difference of a 600- and a 100-iteration call, each the fastest of three
    (setup, first forces and outputs cancel; the call is synchronous and timed
    on the host); the rate is image-site iterations per second.  Algorithmic
    bytes per site and iteration: GNEB field pass m in, F out (48; the
    neighbouring images' spins it also reads come from L2); GNEB force and
    transport m, m_old, F, F_old in (96), F out (24); move m, F in (48), m out
    (24): 240.
    The same path is then held on the deck's plan (mj_gneb_path, key
    `on_plan`), timed the same way.  The CPU baseline is the oracle's find_path
    on one host core on the same path for 20 iterations."""
    import time

    import numpy as np
    import torch

    import matjes_b200 as mj
    from matjes_b200.gneb import geodesic_path
    from oracle import oracle as O

    deck = mj.square_film((side, side, 1), Jv=1e-3, Dv=0.4e-3, Kv=-0.2e-3, Bz=0.3, mu_s=2.0, periodic=(1, 1, 0))
    n = side * side
    up = np.tile([0.0, 0.0, 1.0], (n, 1))
    path = geodesic_path(up, -up, nim, amp_rnd=1e-2, seed=1)
    path[0], path[-1] = up, -up
    path = np.ascontiguousarray(path)
    batch = mj.ReplicaBatch(deck, [(side, side)] * nim, np.tile(deck.B_ext, (nim, 1)), [0.0] * nim, device=dev)

    def call(its):
        batch.upload(path.reshape(-1, 3))
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        r = batch.gneb_path(0.3, 0.02, 1.0, 0.0, its, "I")
        dt = time.perf_counter() - t0
        assert r[3] == its
        return dt

    call(40)
    short = min(call(100) for _ in range(3))
    long_ = min(call(600) for _ in range(3))
    per_it = (long_ - short) / 500
    pk = peaks()
    bpsite = 240.0
    ach = bpsite * n * nim / per_it / 1e9
    del batch
    # the same path held on the deck's plan (mj_gneb_path: one launch of the
    # plan's tiled kernel over all images with the projection and the path sums,
    # then the per-image sums): 240 algorithmic bytes per image site and
    # iteration, as the batch (the GNEB pass 48, the step 120, the move 72); the
    # plan's tile variant autotuned first
    from matjes_b200.gneb import PlanPath

    ham_p = mj.Hamiltonian(deck, device=dev)
    holder = PlanPath(ham_p, path)
    tv = plan_variant_tuned(ham_p, holder.m[0])

    def call_plan(its):
        holder.m.copy_(torch.tensor(path.transpose(0, 2, 1).copy(), device=holder.m.device))
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        r = holder.gneb_path(0.3, 0.02, 1.0, 0.0, its, "I")
        dt = time.perf_counter() - t0
        assert r[3] == its
        return dt

    call_plan(40)
    per_it_plan = (min(call_plan(600) for _ in range(3)) - min(call_plan(100) for _ in range(3))) / 500
    del holder, ham_p
    plan_bpsite = 240.0
    plan_ach = plan_bpsite * n * nim / per_it_plan / 1e9
    mod = O.Model(deck)
    O.set_threads(1)
    try:
        t0 = time.perf_counter()
        O.gneb_find_path(mod, path.copy(), spring=0.3, dt=0.02, mass=1.0, ftol=0.0, itrmax=20, en_zero="I")
        ct = time.perf_counter() - t0
    finally:
        O.set_threads(0)
    return {"workload": f"square{side}_path{nim}_gneb", "sites": n * nim, "images": nim,
            "value": n * nim / per_it, "unit": "image-site iterations/s", "us_per_iteration": 1e6 * per_it,
            "launches_per_iteration": 4,
            "roofline": {"bound": "hbm", "alg_bytes_per_site": bpsite, "achieved": ach, "peak": pk["hbm_gbs"],
                         "unit": "GB/s", "frac": ach / pk["hbm_gbs"], "peak_source": pk["source"]},
            "on_plan": {"path": "mj_gneb_path: the images held on the deck's plan, one tiled launch over all "
                                "images (5D tensor map with an image index) with the projection and the path sums, "
                                "then the per-image sums, step and move",
                        "value": n * nim / per_it_plan, "us_per_iteration": 1e6 * per_it_plan,
                        "launches_per_iteration": 4, "tile_variant": tv,
                        "roofline": {"bound": "hbm", "alg_bytes_per_site": plan_bpsite, "achieved": plan_ach,
                                     "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": plan_ach / pk["hbm_gbs"],
                                     "peak_source": pk["source"]}},
            "cpu_baseline": {"value": n * nim * 20 / ct, "unit": "image-site iterations/s", "cores": 1,
                             "kind": "port",
                             "sample": f"{side}x{side} film, {nim} images, 20 iterations (orc_gneb_find_path, "
                                       f"forces before the first move and outputs included)"}}


class L2Flush:
    """Before every timed step: a 256 MiB write, then a read of another 256 MiB
    buffer, so that the step starts from an L2 (126 MB) that holds none of its
    fields and no dirty lines of the flush (which the step would otherwise
    write back on the flush's behalf)."""

    def __init__(self, device):
        import torch

        self.w = torch.empty(FLUSH_BYTES // 8, dtype=torch.float64, device=device)
        self.r = torch.zeros(FLUSH_BYTES // 8, dtype=torch.float64, device=device)

    def __call__(self):
        self.w.zero_()
        self.r.sum()


def timed_steps(lib, _abi, plan, m, p, first_step, K, flush, E, stream):
    """K single steps of `p` on device spins m, L2 flushed before each; CUDA
    events around each step on the launching stream.  Returns the summed ms."""
    import torch

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    torch.cuda.synchronize()
    for k in range(K):
        flush()
        p.step0 = first_step + k
        ev[k][0].record()
        _abi.check(lib.mj_step_dev(plan, m.data_ptr(), _abi.C.byref(p), 1, E[k:].data_ptr() if E is not None else None,
                                   stream))
        ev[k][1].record()
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev)


OPTION_NAMES = {"fused": 1, "pdl": 2, "store_draw": 3, "blocks_per_sm": 5}  # mj_plan_set_option ids


def tune_kernels(lib, _abi, plan, m, p, flush, E, stream, variants=True):
    """The plan's kernel configuration timed under the bench's own conditions
    (L2 flushed before every step, per-step CUDA events, median of 8): first the
    variant and its halo staging (two launches per step), then, one at a time on
    top of the best, the fused one-launch step, no programmatic dependent launch
    and the redrawn (not stored) Philox draw.  Returns the chosen configuration
    and the table of medians (ms per step)."""
    def med(k0):
        timed_steps(lib, _abi, plan, m, p, k0, 2, flush, E, stream)
        return sorted(timed_steps(lib, _abi, plan, m, p, k0 + 2 + k, 1, flush, E, stream) for k in range(8))[4]

    table = {}
    best = {"variant": None, "tma": None, "fused": 0, "pdl": 1, "store_draw": 1, "blocks_per_sm": 0}
    for name, val in (("fused", 0), ("pdl", 1), ("store_draw", 1), ("blocks_per_sm", 0)):
        _abi.check(lib.mj_plan_set_option(plan, OPTION_NAMES[name], val))
    if variants:
        configs = [(-1, 0)] + [(v, t) for t in (0, 1) for v in range(6)]
        for v, t in configs:
            _abi.check(lib.mj_plan_set_variant(plan, v))
            _abi.check(lib.mj_plan_set_tma(plan, t))
            table["generic" if v < 0 else f"tile{v}" + ("_tma" if t else "")] = med(1000)
        key = min(table, key=table.get)
        bv = -1 if key == "generic" else int(key[4])
        bt = 1 if key.endswith("_tma") else 0
        _abi.check(lib.mj_plan_set_variant(plan, bv))
        _abi.check(lib.mj_plan_set_tma(plan, bt))
        best.update(variant=bv, tma=bt)
    base = min(table.values()) if table else med(1000)
    for name, val in (("fused", 1), ("pdl", 0), ("store_draw", 0), ("blocks_per_sm", 7), ("blocks_per_sm", 6),
                      ("blocks_per_sm", 5)):
        _abi.check(lib.mj_plan_set_option(plan, OPTION_NAMES[name], val))
        t = med(2000)
        table[f"{name}={val}"] = t
        if t < base:
            base = t
            best[name] = val
        else:
            _abi.check(lib.mj_plan_set_option(plan, OPTION_NAMES[name], best[name]))
    return best, {k: round(float(v), 5) for k, v in table.items()}


def kernel_table(prof, bytes_site, N):
    """Per-kernel launches, average time and achieved algorithmic GB/s."""
    out = {}
    for name, (tot, cnt) in prof.items():
        avg = tot / max(cnt, 1)
        b = bytes_site.get(name, 0.0) * N
        out[name] = {"launches": cnt, "avg_us": round(1e3 * avg, 3), "alg_bytes_per_site": bytes_site.get(name),
                     "achieved_gbs": round(b / (avg / 1e3) / 1e9, 1) if b else None}
    return out


def run_integrator_key(dev, wname, integrator, K, W, noise=None, inject_steps=0):
    """The headline workload's lattice, couplings and temperature with another
    integrator or noise source, timed as the headline (L2 flushed before every
    step, CUDA events per step), with the per-kernel split.  Algorithmic bytes
    per site: SIB 48 + 72 (+24 written and read back for the draw at T > 0);
    Matjes Heun 72 + 72 (pass 1 reads m, writes the predictor and D(m_n); pass 2
    reads the predictor and D(m_n), writes m) + 48 for the thermal torque DT
    (written by pass 1, read by pass 2); injected noise: the SIB passes read the
    step's N(0,1) slot (24 B per pass) instead of drawing."""
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi
    from matjes_b200.deck import workload

    w = workload(wname)
    deck, dyn = w["deck"], dict(w["dyn"])
    dyn.pop("steps")
    dyn["integrator"] = integrator
    N = deck.nsites
    ham = mj.Hamiltonian(deck, device=dev)
    buf = None
    if noise == "inject":
        dyn["noise"] = "inject"
        g = torch.Generator(device=f"cuda:{dev}").manual_seed(1)
        buf = torch.randn((inject_steps, 3, N), dtype=torch.float64, device=f"cuda:{dev}", generator=g)
    sd = mj.SpinDynamics(ham, inject=buf, **dyn)
    p = sd.p
    p.energy_mode = _abi.MJ_ENERGY_BEFORE
    m = torch.tensor(w["m0"].T.copy(), device=f"cuda:{dev}")
    lib = _abi.lib
    flush = L2Flush(m.device)
    E = torch.zeros(K + W + 8, dtype=torch.float64, device=m.device)
    stream = torch.cuda.current_stream().cuda_stream
    cfg, _ = tune_kernels(lib, _abi, ham.plan, m, p, flush, E, stream)
    timed_steps(lib, _abi, ham.plan, m, p, 0, W, flush, E, stream)
    ms = timed_steps(lib, _abi, ham.plan, m, p, W, K, flush, E, stream)
    _abi.check(lib.mj_profile_enable(ham.plan, 1))
    timed_steps(lib, _abi, ham.plan, m, p, W + K, K, flush, E, stream)
    prof = _abi.profile_read(ham.plan)
    _abi.check(lib.mj_profile_enable(ham.plan, 0))
    _abi.check(lib.mj_plan_check_status(ham.plan))
    pk = peaks()
    thermal = dyn.get("temperature", 0.0) > 0
    if integrator == "sib":
        extra = 24.0 if (thermal and noise == "inject") else 0.0
        bytes_site = {"k_sib1": 48.0 + extra, "k_sib2": 72.0 + extra, "k_sib_fused": 120.0 + 2 * extra}
        step_b = 120.0 + 2 * extra
    else:
        bytes_site = {"k_heun1": 72.0 + (24.0 if thermal else 0.0), "k_heun2": 72.0 + (24.0 if thermal else 0.0)}
        step_b = sum(bytes_site.values())
    sec = ms / K / 1e3
    return {"workload": wname, "integrator": integrator, "noise": dyn.get("noise", "off"), "kernels_config": cfg,
            "value": N / sec, "unit": UNIT, "ms_per_step": ms / K,
            "step_roofline": {"alg_bytes_per_site": step_b, "achieved_gbs": step_b * N / sec / 1e9,
                              "frac": step_b * N / sec / 1e9 / pk["hbm_gbs"]},
            "kernels": kernel_table(prof, bytes_site, N),
            **({"inject_buffer": f"{inject_steps} steps x 3 x {N} doubles ({buf.numel() * 8 / 1e9:.2f} GB)"}
               if buf is not None else {})}


def run_gpu(args, rank, world):
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi
    from matjes_b200.deck import workload

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    dist = world > 1
    if dist:
        import torch.distributed as td

    w = workload(args.workload)
    deck, dyn = w["deck"], dict(w["dyn"])
    dyn.pop("steps")
    N = deck.nsites
    ham = mj.Hamiltonian(deck, device=dev)
    sd = mj.SpinDynamics(ham, stream_id=replica_stream(rank), **dyn)
    p = sd.p
    p.energy_mode = _abi.MJ_ENERGY_BEFORE
    m = torch.tensor(w["m0"].T.copy(), device=f"cuda:{dev}")
    K, W = args.steps, args.warmup
    E = torch.zeros(W + 2 * K + 16, dtype=torch.float64, device=m.device)
    flush = L2Flush(m.device)
    stream = torch.cuda.current_stream().cuda_stream
    lib = _abi.lib

    # kernel configuration timed under the conditions of the timed loop below
    # (L2 flushed before every step, per-step events); the library's own
    # mj_plan_autotune times back-to-back steps, the right choice when the fields
    # stay in L2 between steps.  --variant fixes it instead (a run under a
    # profiler, whose timing would pick another configuration than a live run).
    if args.variant is None:
        best, tune = tune_kernels(lib, _abi, ham.plan, m, p, flush, E, stream)
    else:
        best = {"variant": args.variant, "tma": args.tma, "fused": args.fused, "pdl": 1, "store_draw": 1}
        _abi.check(lib.mj_plan_set_variant(ham.plan, args.variant))
        _abi.check(lib.mj_plan_set_tma(ham.plan, args.tma))
        _abi.check(lib.mj_plan_set_option(ham.plan, OPTION_NAMES["fused"], args.fused))
        tune = {}

    timed_steps(lib, _abi, ham.plan, m, p, 0, W, flush, E, stream)
    if dist:
        td.barrier()
    clocks = Clocks(dev)
    clocks.start()
    ms = timed_steps(lib, _abi, ham.plan, m, p, W, K, flush, E, stream)
    if dist:
        td.barrier()
    ck = clocks.stop()
    # per-kernel live timing on a second pass of the same K steps
    _abi.check(lib.mj_profile_enable(ham.plan, 1))
    timed_steps(lib, _abi, ham.plan, m, p, W + K, K, flush, E, stream)
    prof = _abi.profile_read(ham.plan)
    _abi.check(lib.mj_profile_enable(ham.plan, 0))
    _abi.check(lib.mj_plan_check_status(ham.plan))
    ms_max = max_over_ranks(ms, m.device, dist)
    value = job_rate(N, K, world, ms_max / 1e3)

    # end to end through the reference-facing host call: mj_step_host takes the
    # pinned host AoS spins, returns the stepped spins in place and the energy.
    # The stripe count of the call is a plan option: short timed sweep, then the
    # measurement with the fastest.
    host = torch.empty((N, 3), dtype=torch.float64, pin_memory=True)
    host.copy_(torch.from_numpy(w["m0"]))
    Eh = np.empty(1)

    def host_steps(n, step0):
        ts = []
        for k in range(n):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            p.step0 = step0 + k
            _abi.check(lib.mj_step_host(ham.plan, host.data_ptr(), _abi.C.byref(p), 1, Eh.ctypes.data))
            _ = float(Eh[0])
            ts.append(time.perf_counter() - t0)
        return ts

    stripe_ms = {}
    for zc in (1, 0):
        _abi.check(lib.mj_plan_set_option(ham.plan, _abi.MJ_OPT_HOST_ZEROCOPY, zc))
        for hs in (2, 3, 4, 6, 8):
            _abi.check(lib.mj_plan_set_option(ham.plan, _abi.MJ_OPT_HOST_STRIPES, hs))
            stripe_ms[f"{hs}{'_zerocopy' if zc else ''}"] = round(
                1e3 * float(np.median(host_steps(10, 20_000 + 100 * hs + 1000 * zc)[2:])), 4)
    best_host = min(stripe_ms, key=stripe_ms.get)
    host_stripes, host_zc = int(best_host.split("_")[0]), int(best_host.endswith("_zerocopy"))
    _abi.check(lib.mj_plan_set_option(ham.plan, _abi.MJ_OPT_HOST_STRIPES, host_stripes))
    _abi.check(lib.mj_plan_set_option(ham.plan, _abi.MJ_OPT_HOST_ZEROCOPY, host_zc))
    host.copy_(torch.from_numpy(w["m0"]))
    ke = max(3, min(K, 20))
    times = host_steps(ke + 2, 10_000)[2:]
    e2e = job_rate(N, len(times), world, max_over_ranks(sum(times), m.device, dist))

    if rank != 0:
        return
    pk = peaks()
    thermal = dyn.get("temperature", 0.0) > 0 and dyn.get("noise") == "philox"
    # algorithmic bytes per site of the SIB step's kernels: the two passes (read
    # m, write the midpoint; read the midpoint and m, write m) or the one fused
    # launch doing both; the stored draw (written by the predictor, read by the
    # corrector at T > 0) is not counted
    bytes_site = {"k_sib1": 48.0, "k_sib2": 72.0, "k_sib_fused": 120.0}
    kernels = kernel_table(prof, bytes_site, N)
    dom = max((k for k in kernels if k in bytes_site), key=lambda k: kernels[k]["avg_us"])
    ach = kernels[dom]["achieved_gbs"]
    tr = ncu_traffic(dom)
    cpu = cpu_oracle_rate(args.workload) if (world == 1 and not args.no_cpu_baseline) else None
    extras = {}
    if world == 1 and not args.no_batch:
        extras["heun"] = run_integrator_key(dev, args.workload, "heun", K, W)
        extras["inject"] = run_integrator_key(dev, args.workload, "sib", K, W, noise="inject", inject_steps=200)
        extras["batch"] = run_batch(dev)
        extras["adjoint"] = run_adjoint(dev)
        extras["dipolar"] = run_dipolar(dev)
        extras["monte_carlo"] = run_monte_carlo(dev)
        extras["hbm_resident_4096"] = run_hbm_resident(dev)
        extras["gneb"] = run_gneb(dev)
    # bulky tables go to stderr, not into the bench line
    verbose = {"kernel_tuning_ms_per_step": tune, "host_stripes_ms_per_step": stripe_ms}
    for k, v in extras.items():
        if isinstance(v, dict) and "autotune_ms_per_step" in v:
            verbose[f"{k}_autotune_ms_per_step"] = v.pop("autotune_ms_per_step")
    sys.stderr.write(json.dumps({"bench_tables": verbose}) + "\n")
    step_frac = 120.0 * N / (ms_max / K / 1e3) / 1e9 / pk["hbm_gbs"]
    line = {
        "metric": metric_name(), "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(args.workload, deck, w["dyn"],
                                                       {"parallelism": f"replicas x{world}" if world > 1 else "single",
                                                        "energy_per_step": ENERGY_CONVENTION}),
        "kernel_config": best,
        "roofline": {"bound": "hbm", "achieved": ach, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": ach / pk["hbm_gbs"], "traffic": None if tr is None else tr * N,
                     # DRAM bytes of the ncu capture over the live launch time, and the
                     # capture's FP64-pipe utilisation of the same kernel
                     "dram_gbs": None if tr is None else round(tr * N / (kernels[dom]["avg_us"] * 1e3), 1),
                     "fp64_pipe_pct": ncu_figure("fp64_pipe_pct", dom),
                     "kernel": dom, "alg_bytes_per_site": bytes_site[dom], "peak_source": pk["source"]},
        "step_roofline": {"alg_bytes_per_site": 120.0, "achieved_gbs": 120.0 * N / (ms_max / K / 1e3) / 1e9,
                          "frac": step_frac, "draw_bytes_per_site": 48.0 if thermal else 0.0},
        "kernels": kernels,
        "clocks": ck,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 24 * N, "d2h_bytes_per_step": 24 * N + 8,
                "path": "mj_step_host: pinned host AoS in and out, one step, energy to the host; copies, "
                        f"transposes and passes overlapped in {host_stripes} stripes of tile rows"
                        + (", the stepped spins written by kernels into the mapped buffer" if host_zc else ""),
                "host_stripes": host_stripes, "host_zerocopy": host_zc},
        "gpu_launches": int(sum(c for _, c in prof.values())),
        "cpu_baseline": cpu,
        **extras,
    }
    # the figures to compare at a glance, last in the line
    summ = {"step_roofline_frac": round(step_frac, 4), "kernel_roofline_frac": round(ach / pk["hbm_gbs"], 4)}
    if extras:
        b, a, d, h, inj = extras["batch"], extras["adjoint"], extras["dipolar"], extras["heun"], extras["inject"]
        summ.update({
            "heun_spin_updates_per_s": h["value"], "heun_step_roofline_frac": round(h["step_roofline"]["frac"], 4),
            "inject_spin_updates_per_s": inj["value"],
            "batch_spin_updates_per_s": b["value"],
            "batch_speedup_vs_sequential_plain": round(b["speedup_vs_sequential_plain"], 3),
            "batch_speedup_vs_sequential_graphs": round(b["speedup_vs_sequential_graphs"], 3),
            "adjoint_cost_ratio": round(a["cost_ratio"], 3),
            "adjoint_cost_ratio_vs_graph_forward": round(a["cost_ratio_vs_graph_forward"], 3),
            "dipolar_spin_updates_per_s": d["value"],
            "dipolar_padded_grid_spin_updates_per_s": d["padded_grid"]["value"],
            "dipolar_eval_roofline_frac": round(d["reference_grid"]["dipolar_eval"]["frac"], 4),
            "hbm_resident_4096_step_roofline_frac": round(extras["hbm_resident_4096"]["step_roofline"]["frac"], 4)})
    if cpu:
        summ["cpu_baseline_spin_updates_per_s"] = cpu["value"]
    line["summary"] = summ
    print(json.dumps(line), flush=True)

# ----------------------------------------------------------------------
# --profile-run: a few launches of a synthetic workload for a profiler (ncu)
# to capture; nothing is timed or printed as a bench line.
PROFILE_RUN_DOC = """Run a few LLG steps of a synthetic workload, for profilers (ncu) to capture.

    python bench.py --profile-run --lattice triangular --L 4096 --T 10 \
        --integrator sib --variant 2 --steps 3

--variant: -1 generic kernel, 0..5 tiled tile shapes, "auto" = the autotuner's pick.

    python bench.py --profile-run --adjoint --L 256 --steps 20 --every 10

runs one forward + backward sweep of the reverse-mode SIB trajectory instead;

    python bench.py --profile-run --batch --steps 3 [--variant 3 --bps 8]

steps the 256-replica batch workload (its configuration autotuned, or the
batch tile variant 0..4 with --bps blocks per SM);

    python bench.py --profile-run --mc --lattice square --L 2048 --steps 3

runs Metropolis sweeps (cone proposals, 10 K) instead of time steps;

    python bench.py --profile-run --gneb --L 256 --nim 16 --steps 64

relaxes a GNEB path of --nim images of an L x L DMI film (J + D + K + Bz =
0.3 T, periodic; geodesic from +z to -z, interior spins moved by up to 1e-2)
for --steps iterations (force tolerance 0); with --plan the images are held on
the deck's plan (mj_gneb_path) instead of as the replicas of a batch.
"""


def _prof_main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--lattice", default="triangular", choices=["triangular", "square", "film"])
    ap.add_argument("--L", type=int, default=4096)
    ap.add_argument("--Lz", type=int, default=16)
    ap.add_argument("--T", type=float, default=10.0)
    ap.add_argument("--integrator", default="sib")
    ap.add_argument("--variant", default="auto")
    ap.add_argument("--bps", type=int, default=8, help="with --batch and a --variant: blocks per SM")
    ap.add_argument("--tma", type=int, default=1, help="halo staging of the tiled kernels: 1 TMA, 0 plain loads")
    ap.add_argument("--fused", type=int, default=0, help="SIB steps: 1 one fused launch, 0 two launches")
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
        return _prof_gneb(a)
    if a.adjoint:
        return _prof_adjoint(a)
    if a.batch:
        return _prof_batch(a)

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
    if ham.noffsets:
        _abi.check(_abi.lib.mj_plan_set_fused(ham.plan, int(a.fused)))
    E = torch.zeros(a.steps + 1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for k in range(a.steps):
        sd.p.step0 = k
        _abi.check(_abi.lib.mj_step_dev(ham.plan, m.data_ptr(), _abi.C.byref(sd.p), 1, E[k:].data_ptr(), stream))
    torch.cuda.synchronize()
    print("ok", E[: a.steps].tolist())


def _prof_adjoint(a):
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


def plan_variant_tuned(ham, m_soa) -> int:
    """The plan's tile variant autotuned on SIB steps of the spins m_soa (a (3,
    N) device tensor, left untouched); -1 for a plan without tiled kernels."""
    import matjes_b200 as mj
    from matjes_b200 import _abi

    tv = _abi.C.c_int32(-1)
    if ham.noffsets:
        sd = mj.SpinDynamics(ham, integrator="sib", timestep=0.1, alpha=0.1)
        _abi.check(_abi.lib.mj_plan_autotune(ham.plan, m_soa.data_ptr(), _abi.C.byref(sd.p), 3, _abi.C.byref(tv),
                                             None, None))
    return int(tv.value)


def _prof_gneb(a):
    import matjes_b200 as mj
    from matjes_b200.gneb import geodesic_path

    deck = mj.square_film((a.L, a.L, 1), Jv=1e-3, Dv=0.4e-3, Kv=-0.2e-3, Bz=0.3, mu_s=2.0, periodic=(1, 1, 0))
    n = a.L * a.L
    up = np.tile([0.0, 0.0, 1.0], (n, 1))
    path = geodesic_path(up, -up, a.nim, amp_rnd=1e-2, seed=1)
    path[0], path[-1] = up, -up
    if a.plan:
        from matjes_b200.gneb import PlanPath

        ham = mj.Hamiltonian(deck)
        bt = PlanPath(ham, path)
        plan_variant_tuned(ham, bt.m[0])
    else:
        bt = mj.ReplicaBatch(deck, [(a.L, a.L)] * a.nim, np.tile(deck.B_ext, (a.nim, 1)), [0.0] * a.nim)
        bt.upload(path.reshape(-1, 3))
    rx, ene, dene, its, fchk, _ = bt.gneb_path(0.3, 0.02, 1.0, 0.0, a.steps, "I")
    print("ok", its, fchk, ene.tolist())


def _prof_batch(a):
    import torch

    import matjes_b200 as mj

    w = mj.workload("square_replicas256")
    bt = mj.ReplicaBatch(w["cell"], w["sizes"], w["B_ext"], w["temperature"])
    bt.upload(w["m0"])
    d = w["dyn"]
    p = bt.params(timestep=d["timestep"], alpha=d["alpha"], noise="philox", seed=d["seed"])
    if a.variant == "auto":
        bt.autotune(p, steps=5)  # the configuration the bench's batch key runs
    else:  # a fixed configuration (the autotuner's timing under a profiler picks another)
        bt.set_config(int(a.variant), a.bps)
    bt.upload(w["m0"])
    bt.step(p, a.steps)
    torch.cuda.synchronize()
    print("ok", bt.energies()[:4].tolist())


def main():
    # every oracle import of this process (the CPU legs) loads the build made on this host
    os.environ["ORACLE_NATIVE"] = "1"
    if "--profile-run" in sys.argv[1:]:
        argv = [a for a in sys.argv[1:] if a != "--profile-run"]
        _prof_main(argv)
        return
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="triangular1024_thermal")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variant", type=int, default=None,
                    help="kernel variant (-1 generic, 0..5 tiled) instead of the timed sweep")
    ap.add_argument("--tma", type=int, default=0, help="halo staging with --variant: 1 TMA, 0 plain loads")
    ap.add_argument("--fused", type=int, default=0, help="with --variant: 1 one launch per SIB step, 0 two")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batch, adjoint, dipolar and Monte Carlo measurements")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_gpu(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as td

            td.destroy_process_group()


if __name__ == "__main__":
    main()
