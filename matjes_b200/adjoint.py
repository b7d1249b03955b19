"""Reverse mode of the SIB trajectory as a torch.autograd.Function (mj_adjoint_*).

``SIBTrajectory(ham, nsteps, ...)(m0, terms, bfield)`` returns the spins after
``nsteps`` SIB steps (device SoA (3, N), float64) and differentiates them with
respect to the initial spins ``m0``, the coupling-term values ``terms`` (the
J, D and K terms of the deck in that order, eV, with the reference's input
sign) and the per-site applied field ``bfield`` ((3, N) T, or None for the
deck's uniform field).  The forward map is the reference's dynamics loop
(dynamics/spindynamics.f90:282-313) with the SIB scheme of Mentink et al.
(2010); the backward sweep is the hand-written transpose in mj_adjoint.cu,
with checkpoints every ``checkpoint_every`` steps.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _abi
from ._abi import check, lib, ptr
from .hamiltonian import Hamiltonian


def _stream(t) -> int:
    import torch

    return torch.cuda.current_stream(t.device).cuda_stream


def deck_terms(deck) -> np.ndarray:
    """The term values of a deck in the plan's order: J terms, D terms, K terms."""
    return np.array([t[-1] for t in deck.J] + [t[-1] for t in deck.D] + [t[-1] for t in deck.K], np.float64)


def field_vjp(ham: Hamiltonian, m, v):
    """(dB/dm)^T v, dB/dvalue_t . v, (dB/db)^T v of the plan's field at m (device SoA tensors)."""
    import torch

    n = C.c_int32()
    check(lib.mj_plan_nterms(ham.plan, C.byref(n)))
    gm = torch.empty_like(m)
    gb = torch.empty_like(m)
    gt = torch.zeros(max(1, n.value), dtype=torch.float64, device=m.device)
    check(lib.mj_field_vjp(ham.plan, ptr(m), ptr(v), ptr(gm), ptr(gt) if n.value else None, ptr(gb), _stream(m)))
    return gm, gt[:n.value], gb


class SIBTrajectory:
    def __init__(self, ham: Hamiltonian, nsteps: int, checkpoint_every: int = 50, timestep: float = 0.1,
                 alpha: float = 0.2, temperature: float = 0.0, noise: str = "off", seed: int = 0, stream_id: int = 0,
                 step0: int = 0):
        self.ham = ham
        self.nsteps = int(nsteps)
        n = C.c_int32()
        check(lib.mj_plan_nterms(ham.plan, C.byref(n)))
        self.nterms = int(n.value)
        h = C.c_void_p()
        check(lib.mj_adjoint_create(ham.plan, self.nsteps, int(checkpoint_every), C.byref(h)))
        self.handle = h
        self.p = _abi.DynParams()
        self.p.integrator = _abi.MJ_SIB
        self.p.timestep = float(timestep)
        self.p.alpha = float(alpha)
        self.p.temperature = float(temperature)
        self.p.noise = _abi.NOISES[noise]
        self.p.seed = int(seed)
        self.p.stream_id = int(stream_id)
        self.p.step0 = int(step0)
        self._terms = None if ham.deck is None else deck_terms(ham.deck)
        self._forward_id = 0
        self._last = None

    # -- plan parameters ---------------------------------------------------
    def set_terms(self, values) -> None:
        v = np.ascontiguousarray(np.asarray(values, np.float64).reshape(-1))
        assert v.size == self.nterms
        if self._terms is None or not np.array_equal(v, self._terms):
            check(lib.mj_plan_set_terms(self.ham.plan, ptr(v)))
            self._terms = v.copy()

    def set_bfield(self, b) -> None:
        """Per-site applied field, a (3, N) CUDA tensor (T)."""
        assert b.is_cuda and b.is_contiguous() and b.shape == (3, self.ham.N)
        check(lib.mj_plan_set_bfield_device(self.ham.plan, ptr(b), _stream(b)))

    # -- raw forward / backward -------------------------------------------
    def forward(self, m0):
        import torch

        m0 = m0.contiguous()
        mT = torch.empty_like(m0)
        check(lib.mj_adjoint_forward(self.handle, C.byref(self.p), ptr(m0), ptr(mT), _stream(m0)))
        self._forward_id += 1
        return mT

    def backward(self, gT, want_b: bool = True):
        import torch

        gT = gT.contiguous()
        g0 = torch.empty_like(gT)
        gt = torch.zeros(max(1, self.nterms), dtype=torch.float64, device=gT.device)
        gb = torch.empty_like(gT) if want_b else None
        check(lib.mj_adjoint_backward(self.handle, ptr(gT), ptr(g0), ptr(gt) if self.nterms else None, ptr(gb),
                                      _stream(gT)))
        return g0, gt[:self.nterms], gb

    def __call__(self, m0, terms=None, bfield=None):
        return _SIBFn.apply(m0, terms, bfield, self)

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.mj_adjoint_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _load_inputs(traj: SIBTrajectory, terms, bfield):
    if terms is not None:
        traj.set_terms(terms.detach().cpu().numpy())
    if bfield is not None:
        traj.set_bfield(bfield.detach().contiguous())


try:
    import torch

    class _SIBFn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, m0, terms, bfield, traj):
            _load_inputs(traj, terms, bfield)
            mT = traj.forward(m0.detach())
            ctx.traj = traj
            ctx.fid = traj._forward_id
            ctx.has_terms = terms is not None
            ctx.has_b = bfield is not None
            ctx.save_for_backward(m0.detach(), terms if terms is not None else torch.empty(0),
                                  bfield if bfield is not None else torch.empty(0))
            return mT

        @staticmethod
        def backward(ctx, gT):
            traj = ctx.traj
            m0, terms, bfield = ctx.saved_tensors
            if traj._forward_id != ctx.fid:  # another forward ran since: rebuild this one's checkpoints
                _load_inputs(traj, terms if ctx.has_terms else None, bfield if ctx.has_b else None)
                traj.forward(m0)
            g0, gt, gb = traj.backward(gT, want_b=ctx.has_b)
            gterms = gt.to(terms.device) if ctx.has_terms else None
            return g0, gterms, gb, None
except ImportError:  # torch is needed only for the autograd entry point
    _SIBFn = None
