"""Batched replicas with parallel tempering over the C ABI (mj_batch_*).

A ``ReplicaBatch`` holds many independent 2D lattices of one single-atom
Hamiltonian (the cell, shells and couplings of a ``Deck``), each with its own
size, applied field and temperature, advanced together by SIB.  In the
reference every replica is a separate run of dynamics/spindynamics.f90:260-323
(one per MPI rank group in paratemp-MC/parallel_tempering.f90:24-217); the
temperature swaps follow paratemp-MC/paratemp.f90:47-119.

Host arrays use the reference AoS layout (Ntot, 3) in replica order; the
device state is SoA (3, Ntot), replica r at columns offsets[r]:offsets[r+1].
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._abi import check, lib, ptr
from .deck import Deck

N_BATCH_VARIANTS = 5
BATCH_BLOCKS_PER_SM = (2, 4, 8, 16, 32)


class ReplicaBatch:
    def __init__(self, cell: Deck, sizes: Sequence[Sequence[int]], B_ext: np.ndarray, temperature: Sequence[float],
                 device: int = 0):
        """cell: the deck whose cell and couplings every replica shares (its L and
        B_ext are ignored); sizes: (nrep, 2) lattice sides; B_ext: (nrep, 3) T;
        temperature: (nrep,) K."""
        self.cell = cell
        self.device = device
        L = np.ascontiguousarray(sizes, np.int32).reshape(-1, 2)
        self.nrep = L.shape[0]
        B = np.ascontiguousarray(B_ext, np.float64).reshape(self.nrep, 3)
        T = np.ascontiguousarray(temperature, np.float64).reshape(self.nrep)
        lat, h, keep = cell.c_structs()
        b = C.c_void_p()
        check(lib.mj_batch_create(C.byref(lat), C.byref(h), self.nrep, ptr(L), ptr(B), ptr(T), device, C.byref(b)))
        self._keep = keep
        self.handle = b
        self.sizes = L.copy()
        self.B_ext = B.copy()
        self.T0 = T.copy()
        tot = C.c_int64()
        off = np.zeros(self.nrep + 1, np.int64)
        check(lib.mj_batch_nsites(b, C.byref(tot), ptr(off)))
        self.N = int(tot.value)
        self.offsets = off

    # -- state ------------------------------------------------------------
    def upload(self, m: np.ndarray) -> None:
        mh = np.ascontiguousarray(m, np.float64)
        assert mh.shape == (self.N, 3)
        check(lib.mj_batch_upload(self.handle, ptr(mh), None))

    def download(self) -> np.ndarray:
        out = np.empty((self.N, 3))
        check(lib.mj_batch_download(self.handle, ptr(out), None))
        return out

    def replica(self, m: np.ndarray, r: int) -> np.ndarray:
        """Rows of replica r in a (Ntot, 3) array."""
        return m[self.offsets[r]:self.offsets[r + 1]]

    def device_tensor(self):
        """torch view (3, Ntot) of the batch's device spins (no copy)."""
        from .hamiltonian import _wrap_device

        p = C.c_void_p()
        check(lib.mj_batch_device_ptr(self.handle, C.byref(p)))
        return _wrap_device(p.value, (3, self.N), self.device)

    # -- dynamics ---------------------------------------------------------
    @staticmethod
    def params(timestep: float = 0.1, alpha: float = 0.5, noise: str = "philox", seed: int = 0, stream_id: int = 0,
               step0: int = 0) -> _abi.DynParams:
        p = _abi.DynParams()
        p.integrator = _abi.MJ_SIB
        p.timestep = float(timestep)
        p.alpha = float(alpha)
        p.noise = _abi.NOISES[noise]
        p.seed = int(seed)
        p.stream_id = int(stream_id)
        p.step0 = int(step0)
        return p

    def step(self, p: _abi.DynParams, nsteps: int, swap_every: int = 0, energies: bool = False, stream=None):
        """nsteps SIB steps (p.step0 advances); a parallel-tempering round after
        every step s with (s+1) % swap_every == 0.  Returns the replica energies
        after the last step (a device tensor) when asked."""
        E = None
        if energies:
            import torch

            E = torch.empty(self.nrep, dtype=torch.float64, device=f"cuda:{self.device}")
        check(lib.mj_batch_step(self.handle, C.byref(p), int(nsteps), int(swap_every), ptr(E), stream))
        p.step0 += int(nsteps)
        return E

    def graph_run(self, p: _abi.DynParams, steps_per_graph: int, nreplay: int, swap_every: int = 0, stream=None):
        """The same steps as one CUDA graph of steps_per_graph steps replayed nreplay times."""
        check(lib.mj_batch_graph_run(self.handle, C.byref(p), int(steps_per_graph), int(nreplay), int(swap_every),
                                     None, stream))
        p.step0 += int(steps_per_graph) * int(nreplay)

    def field(self, project: bool = False, energies: bool = True):
        """Effective field of every replica at the current state (device (3, Ntot)),
        optionally with the component along m removed, and the replica energies."""
        import torch

        dev = f"cuda:{self.device}"
        B = torch.empty((3, self.N), dtype=torch.float64, device=dev)
        E = torch.empty(self.nrep, dtype=torch.float64, device=dev) if energies else None
        check(lib.mj_batch_field(self.handle, ptr(B), ptr(E), int(bool(project)), None))
        return B, E

    def gneb_tangent(self, E=None, mode: str = "energy"):
        """Path tangents with the replicas as the images of a path (device (3, Ntot)):
        mode 'energy' (energy-weighted, needs the image energies E) or 'central'."""
        import torch

        tau = torch.empty((3, self.N), dtype=torch.float64, device=f"cuda:{self.device}")
        m = {"energy": 0, "central": 1}[mode]
        check(lib.mj_batch_gneb_tangent(self.handle, ptr(E), m, ptr(tau), None))
        return tau

    def gneb_path(self, spring: float = 0.5, dt: float = 1.0e-2, mass: float = 1.0, ftol: float = 1.0e-3,
                  itrmax: int = 2 ** 62, en_zero: str = "N", climb: bool = False):
        """GNEB relaxation of the path the replicas hold (GNEB/gneb_utils.f90
        find_path; climb: the climbing-image run); the batch is left holding the
        relaxed path.  Returns (rx, ene, dene, iterations, max |F|, climbing
        image or -1)."""
        if en_zero not in ("I", "F", "N"):
            raise ValueError("en_zero is 'I', 'F' or 'N'")
        p = _abi.GnebParams(float(spring), float(dt), float(mass), float(ftol), int(itrmax), ord(en_zero),
                            int(bool(climb)))
        rx, ene, dene = np.zeros(self.nrep), np.zeros(self.nrep), np.zeros(self.nrep)
        it, fc, ci = C.c_int64(), C.c_double(), C.c_int32()
        check(lib.mj_batch_gneb_path(self.handle, C.byref(p), ptr(rx), ptr(ene), ptr(dene), C.byref(it),
                                     C.byref(fc), C.byref(ci)))
        return rx, ene, dene, int(it.value), float(fc.value), int(ci.value)

    def energies(self) -> np.ndarray:
        out = np.empty(self.nrep)
        check(lib.mj_batch_energies(self.handle, ptr(out)))
        return out

    def temperatures(self):
        """(temperature of every replica in K, accepted swaps of every ladder pair)."""
        T = np.empty(self.nrep)
        acc = np.zeros(self.nrep, np.int32)
        check(lib.mj_batch_temperatures(self.handle, ptr(T), ptr(acc)))
        return T, acc

    # -- Monte Carlo -------------------------------------------------------
    def monte_carlo(self, p: _abi.McParams, nrounds: int, sweeps_per_round: int = 1, swap: bool = True,
                    record: bool = True, stream=None):
        """Parallel-tempering Monte Carlo (mj_batch_mc): nrounds rounds of
        sweeps_per_round Metropolis sweeps of every replica, each round measured
        and followed by a swap round when `swap`.  p (McParams) carries the
        proposal, cone, seed, stream base and the advancing sweep and round
        counters.  Returns (E (nrounds, nrep), summed spins (nrounds, nrep, 3),
        ladder slots (nrounds, nrep)) as CUDA tensors (None when not recorded)."""
        import torch

        dev = f"cuda:{self.device}"
        E = torch.empty((nrounds, self.nrep), dtype=torch.float64, device=dev) if record else None
        M = torch.empty((nrounds, self.nrep, 3), dtype=torch.float64, device=dev) if record else None
        S = torch.empty((nrounds, self.nrep), dtype=torch.int32, device=dev) if record else None
        col = np.zeros(4, np.int32)
        check(lib.mj_batch_mc(self.handle, C.byref(p), int(nrounds), int(sweeps_per_round), int(bool(swap)), ptr(E),
                              ptr(M), ptr(S), col.ctypes.data_as(C.POINTER(C.c_int32)), stream))
        self.mc_colors = tuple(int(c) for c in col)
        return E, M, S

    def mc_reset(self, cone: float) -> None:
        check(lib.mj_batch_mc_reset(self.handle, float(cone)))

    def mc_state(self):
        """(cone, accepted moves, proposed moves) of every replica's chain."""
        cone = np.empty(self.nrep)
        acc = np.empty(self.nrep, np.int64)
        prop = np.empty(self.nrep, np.int64)
        check(lib.mj_batch_mc_state(self.handle, ptr(cone), ptr(acc), ptr(prop)))
        return cone, acc, prop

    def set_config(self, variant: int, blocks_per_sm: int) -> None:
        check(lib.mj_batch_set_config(self.handle, int(variant), int(blocks_per_sm)))

    def autotune(self, p: _abi.DynParams, steps: int = 5):
        """Pick the fastest (tile variant, blocks per SM); returns it and the ms/step table."""
        v = C.c_int32()
        bps = C.c_int32()
        table = np.full(N_BATCH_VARIANTS * len(BATCH_BLOCKS_PER_SM), np.nan)
        check(lib.mj_batch_autotune(self.handle, C.byref(p), int(steps), C.byref(v), C.byref(bps), ptr(table)))
        return (int(v.value), int(bps.value)), table.reshape(N_BATCH_VARIANTS, len(BATCH_BLOCKS_PER_SM))

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.mj_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

