"""Host-side mirror of Matjes' Hamiltonian and dynamics interface over the C ABI.

``Hamiltonian`` stands in for ``type(hamiltonian)``
(Hamiltonian_type/hamiltonian_collection.f90:15-60): ``get_eff_field``
(:433-454), ``energy`` (:390-400) and ``energy_distrib`` (:332-363), with the
same argument meaning (field = -dE/dm in eV, per-site energies left-assigned).
``SpinDynamics`` stands in for the step loop of dynamics/spindynamics.f90:260-323.

Arrays on the host use the reference AoS layout (N, 3); arrays on the device
(torch CUDA tensors) use the kernels' SoA layout (3, N) and are passed by
pointer on torch's current stream.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _abi
from ._abi import check, lib, ptr
from .deck import Deck


def _stream(t) -> Optional[int]:
    import torch

    return torch.cuda.current_stream(t.device).cuda_stream


def _is_torch(x) -> bool:
    return hasattr(x, "data_ptr") and hasattr(x, "is_cuda")


class Hamiltonian:
    def __init__(self, deck: Deck, device: int = 0):
        self.deck = deck
        self.device = device
        lat, h, keep = deck.c_structs()
        plan = C.c_void_p()
        check(lib.mj_plan_create(C.byref(lat), C.byref(h), device, C.byref(plan)))
        self._keep = keep
        self.plan = plan
        n = C.c_int64()
        check(lib.mj_plan_nsites(plan, C.byref(n)))
        self.N = int(n.value)
        self.ncell = deck.ncell

    @classmethod
    def from_coo(cls, nsites, rows, cols, vals, base=0, zeeman=None, b_site=None, device=0):
        """ELL plan from the combined MM matrix in COO form (cuda_H_init input)."""
        self = cls.__new__(cls)
        self.deck = None
        self.device = device
        rows = np.ascontiguousarray(rows, np.int64)
        cols = np.ascontiguousarray(cols, np.int64)
        vals = np.ascontiguousarray(vals, np.float64)
        z = None if zeeman is None else np.ascontiguousarray(zeeman, np.float64)
        b = None if b_site is None else np.ascontiguousarray(b_site, np.float64)
        plan = C.c_void_p()
        check(lib.mj_plan_from_coo(int(nsites), len(vals), ptr(rows), ptr(cols), ptr(vals), int(base), ptr(z), ptr(b),
                                   device, C.byref(plan)))
        self.plan = plan
        self._keep = ()
        self.N = int(nsites)
        self.ncell = int(nsites)
        return self

    def close(self) -> None:
        if getattr(self, "plan", None):
            lib.mj_plan_destroy(self.plan)
            self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def noffsets(self) -> int:
        n = C.c_int32()
        check(lib.mj_plan_noffsets(self.plan, C.byref(n)))
        return int(n.value)

    # ------------------------------------------------------------------
    def set_bfield(self, b_cell) -> None:
        """Per-cell applied field in Tesla ((ncell, 3) host array, or a (3, ncell)
        CUDA tensor); None restores the uniform H_ext."""
        if b_cell is None:
            check(lib.mj_plan_set_bfield(self.plan, None))
        elif _is_torch(b_cell):
            check(lib.mj_plan_set_bfield_device(self.plan, ptr(b_cell.contiguous()), _stream(b_cell)))
        else:
            b = np.ascontiguousarray(b_cell, np.float64)
            assert b.shape == (self.ncell, 3)
            check(lib.mj_plan_set_bfield(self.plan, ptr(b)))

    def get_eff_field(self, m, with_energy: bool = False):
        """B_eff = -dE/dm.  Host (N,3) in -> host (N,3) out; CUDA (3,N) in -> CUDA (3,N) out."""
        if _is_torch(m):
            import torch

            m = m.contiguous()
            B = torch.empty_like(m)
            e = torch.empty(self.N, dtype=m.dtype, device=m.device) if with_energy else None
            check(lib.mj_field_dev(self.plan, ptr(m), ptr(B), ptr(e), _stream(m)))
            return (B, e) if with_energy else B
        mh = np.ascontiguousarray(m, np.float64)
        assert mh.shape == (self.N, 3)
        B = np.empty_like(mh)
        e = np.empty(self.N) if with_energy else None
        check(lib.mj_field_host(self.plan, ptr(mh), ptr(B), ptr(e)))
        return (B, e) if with_energy else B

    def energy_distrib(self, m):
        return self.get_eff_field(m, with_energy=True)[1]

    def energy(self, m) -> float:
        st = SpinState(self, m)
        E = C.c_double()
        check(lib.mj_energy(self.plan, st.handle, C.byref(E)))
        return float(E.value)


class SpinState:
    """Device-resident spin field (mj_state) of a plan."""

    def __init__(self, ham: Hamiltonian, m=None):
        self.ham = ham
        h = C.c_void_p()
        check(lib.mj_state_create(ham.plan, C.byref(h)))
        self.handle = h
        if m is not None:
            self.upload(m)

    def upload(self, m) -> None:
        if _is_torch(m):
            import torch

            assert m.shape == (3, self.ham.N)
            dst = self.device_tensor()
            dst.copy_(m)
            return
        mh = np.ascontiguousarray(m, np.float64)
        assert mh.shape == (self.ham.N, 3)
        check(lib.mj_state_upload(self.handle, ptr(mh), None))

    def download(self) -> np.ndarray:
        out = np.empty((self.ham.N, 3))
        check(lib.mj_state_download(self.handle, ptr(out), None))
        return out

    def device_ptr(self) -> int:
        p = C.c_void_p()
        check(lib.mj_state_device_ptr(self.handle, C.byref(p)))
        return p.value

    def device_tensor(self):
        """A torch view (3, N) of the state's device memory (no copy)."""
        return _wrap_device(self.device_ptr(), (3, self.ham.N), self.ham.device)

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.mj_state_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _wrap_device(addr: int, shape, device: int):
    """Non-owning torch tensor over device memory owned by the library."""
    import torch

    class _Holder:
        pass

    h = _Holder()
    n = int(np.prod(shape))
    h.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (addr, False), "version": 3, "strides": None}
    with torch.cuda.device(device):
        t = torch.as_tensor(h, device=f"cuda:{device}")
    return t.view(*shape)


class SpinDynamics:
    """LLG integration (dynamics/spindynamics.f90:260-323) on the GPU.

    integrator: 'euler' | 'heun' (Matjes Heun, stage dt = timestep/2, corrector
    restarted from the predictor) | 'sib' (Mentink et al. 2010);
    noise: 'off' | 'philox' (seed) | 'inject' (device N(0,1) buffer [nbuf][3][N]).
    """

    def __init__(self, ham: Hamiltonian, integrator: str = "sib", timestep: float = 0.1, alpha: float = 0.1,
                 temperature: float = 0.0, noise: str = "off", seed: int = 0, stream_id: int = 0, inject=None,
                 **_ignored):
        self.ham = ham
        self.p = _abi.DynParams()
        self.p.integrator = _abi.INTEGRATORS[integrator]
        self.p.timestep = float(timestep)
        self.p.alpha = float(alpha)
        self.p.temperature = float(temperature)
        self.p.noise = _abi.NOISES[noise]
        self.p.seed = int(seed)
        self.p.stream_id = int(stream_id)
        self.p.step0 = 0
        self.inject = inject
        if inject is not None:
            assert _is_torch(inject) and inject.is_cuda and inject.shape[1:] == (3, ham.N)
            self.p.inject = ptr(inject)
            self.p.inject_nbuf = int(inject.shape[0])

    def run(self, m, nsteps: int, energies: bool = False, step0: Optional[int] = None):
        """Advance `m` by nsteps.  Host (N,3) arrays are updated in place through
        mj_step_host; CUDA (3,N) tensors in place through mj_step_dev.  Returns
        the per-step energies (after each step) when asked."""
        if step0 is not None:
            self.p.step0 = int(step0)
        if _is_torch(m):
            import torch

            assert m.is_contiguous() and m.shape == (3, self.ham.N)
            E = torch.empty(nsteps, dtype=torch.float64, device=m.device) if energies else None
            check(lib.mj_step_dev(self.ham.plan, ptr(m), C.byref(self.p), int(nsteps), ptr(E), _stream(m)))
        else:
            assert isinstance(m, np.ndarray) and m.dtype == np.float64 and m.flags.c_contiguous
            E = np.empty(nsteps) if energies else None
            check(lib.mj_step_host(self.ham.plan, ptr(m), C.byref(self.p), int(nsteps), ptr(E)))
        self.p.step0 += int(nsteps)
        return E


def minimize(ham: Hamiltonian, m, method: str = "vpo", timestep: float = 0.1, mass: float = 1.0,
             conv_torque: float = 1e-6, max_iter: int = 100000, check_every: int = 100):
    """Energy minimisation on the device (solvers/minimize.F90): method 'vpo'
    (minimize_run, velocity projection) or 'infdamp' (minimize_infdamp_run,
    spins turned onto their local field, colour by colour).  m: a CUDA (3, N)
    tensor, updated in place.  Returns (iterations, max torque[, colours])."""
    assert _is_torch(m) and m.is_contiguous() and m.shape == (3, ham.N)
    p = _abi.MinParams(float(timestep), float(mass), float(conv_torque), int(check_every))
    it, mt = C.c_int64(), C.c_double()
    if method == "vpo":
        check(lib.mj_minimize(ham.plan, ptr(m), C.byref(p), int(max_iter), C.byref(it), C.byref(mt), _stream(m)))
        return it.value, mt.value
    colors = np.zeros(3, np.int32)
    check(lib.mj_minimize_infdamp(ham.plan, ptr(m), C.byref(p), int(max_iter), C.byref(it), C.byref(mt),
                                  colors.ctypes.data, _stream(m)))
    return it.value, mt.value, tuple(int(c) for c in colors)
