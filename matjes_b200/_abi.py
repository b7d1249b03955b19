"""ctypes binding of ``include/matjes_gpu.h`` (the C ABI of the CUDA library).

The shared library ``libmatjes_b200.so`` is built in-tree by
``matjes_b200.build``.  There is no CPU fallback: importing this module
without the built library raises ``ImportError``.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmatjes_b200.so")

MJ_OK = 0
MJ_ERR_ARG = 1
MJ_ERR_OOM = 2
MJ_ERR_CUDA = 3
MJ_ERR_TIMEOUT = 4
MJ_ERR_NAN = 5
MJ_ERR_UNSUPPORTED = 6
MJ_ERR_GEOMETRY = 7

MJ_EULER = 1
MJ_HEUN_MATJES = 2
MJ_SIB = 3
MJ_NOISE_OFF = 0
MJ_NOISE_PHILOX = 1
MJ_NOISE_INJECT = 2
MJ_MAX_ATOMS = 16
MJ_OPT_TMA, MJ_OPT_FUSED, MJ_OPT_PDL, MJ_OPT_STORE_DRAW, MJ_OPT_HOST_STRIPES, MJ_OPT_BLOCKS_PER_SM = 0, 1, 2, 3, 4, 5
MJ_OPT_DIP_ZCONV, MJ_OPT_HOST_ZEROCOPY = 6, 7

INTEGRATORS = {"euler": MJ_EULER, "heun": MJ_HEUN_MATJES, "heun_matjes": MJ_HEUN_MATJES, "sib": MJ_SIB}
NOISES = {"off": MJ_NOISE_OFF, "philox": MJ_NOISE_PHILOX, "inject": MJ_NOISE_INJECT}


class LatticeDesc(C.Structure):
    _fields_ = [
        ("L", C.c_int32 * 3),
        ("periodic", C.c_int32 * 3),
        ("areal", (C.c_double * 3) * 3),
        ("natom", C.c_int32),
        ("frac", (C.c_double * 3) * MJ_MAX_ATOMS),
        ("attype", C.c_int32 * MJ_MAX_ATOMS),
        ("moment", C.c_double * MJ_MAX_ATOMS),
    ]


class ExchangeTerm(C.Structure):
    _fields_ = [("t1", C.c_int32), ("t2", C.c_int32), ("shell", C.c_int32), ("value", C.c_double)]


class DmiTerm(C.Structure):
    _fields_ = [("t1", C.c_int32), ("t2", C.c_int32), ("tmed", C.c_int32), ("shell", C.c_int32), ("value", C.c_double)]


class AnisoTerm(C.Structure):
    _fields_ = [("type", C.c_int32), ("axis", C.c_double * 3), ("value", C.c_double)]


class HamiltonianDesc(C.Structure):
    _fields_ = [
        ("nJ", C.c_int32), ("J", C.POINTER(ExchangeTerm)),
        ("nD", C.c_int32), ("D", C.POINTER(DmiTerm)),
        ("nK", C.c_int32), ("K", C.POINTER(AnisoTerm)),
        ("c_H_J", C.c_double), ("c_H_D", C.c_double), ("c_H_ani", C.c_double), ("c_zeeman", C.c_double),
        ("B_ext", C.c_double * 3),
        ("zeeman_on", C.c_int32),
        ("dip_on", C.c_int32),
        ("dip_period_cut", C.c_int32 * 3),
    ]


class DynParams(C.Structure):
    _fields_ = [
        ("integrator", C.c_int32),
        ("timestep", C.c_double),
        ("alpha", C.c_double),
        ("temperature", C.c_double),
        ("noise", C.c_int32),
        ("seed", C.c_uint64),
        ("stream_id", C.c_uint32),
        ("step0", C.c_uint32),
        ("inject", C.c_void_p),
        ("inject_nbuf", C.c_int32),
        ("energy_mode", C.c_int32),
    ]


class MinParams(C.Structure):
    _fields_ = [("timestep", C.c_double), ("mass", C.c_double), ("conv_torque", C.c_double),
                ("check_every", C.c_int32)]


class McParams(C.Structure):
    _fields_ = [("temperature", C.c_double), ("cone", C.c_double), ("proposal", C.c_int32),
                ("adapt_cone", C.c_int32), ("seed", C.c_uint64), ("stream_id", C.c_uint32),
                ("sweep0", C.c_uint32), ("accepted_total", C.c_int64), ("proposed_total", C.c_int64),
                ("round0", C.c_uint32), ("track_totals", C.c_int32)]


class GnebParams(C.Structure):
    _fields_ = [("spring", C.c_double), ("dt", C.c_double), ("mass", C.c_double), ("ftol", C.c_double),
                ("itrmax", C.c_int64), ("en_zero", C.c_int32), ("climb", C.c_int32)]


MJ_MC_CONE = 0
MJ_MC_ISING = 1
MJ_MC_UNDERRELAX = 2
MJ_MC_OVERRELAX = 3

MJ_ENERGY_AFTER = 0
MJ_ENERGY_BEFORE = 1


class MatjesError(RuntimeError):
    """A C-ABI call returned a non-zero mj_status."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"mj_status {status}: {msg}")
        self.status = status


P = C.c_void_p
DP = C.POINTER(C.c_double)

# name -> (restype, argtypes); every entry is declared in include/matjes_gpu.h
SIGNATURES = {
    "mj_last_error": (C.c_char_p, []),
    "mj_version": (C.c_char_p, []),
    "mj_plan_create": (C.c_int32, [C.POINTER(LatticeDesc), C.POINTER(HamiltonianDesc), C.c_int32, C.POINTER(P)]),
    "mj_stencil_describe": (C.c_int32, [C.POINTER(LatticeDesc), C.POINTER(HamiltonianDesc), C.c_int32,
                                        C.POINTER(C.c_int32), P, P, P, P]),
    "mj_plan_from_coo": (C.c_int32, [C.c_int64, C.c_int64, P, P, P, C.c_int32, P, P, C.c_int32, C.POINTER(P)]),
    "mj_plan_destroy": (C.c_int32, [P]),
    "mj_plan_nsites": (C.c_int32, [P, C.POINTER(C.c_int64)]),
    "mj_plan_noffsets": (C.c_int32, [P, C.POINTER(C.c_int32)]),
    "mj_plan_set_variant": (C.c_int32, [P, C.c_int32]),
    "mj_plan_get_variant": (C.c_int32, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "mj_plan_autotune": (C.c_int32, [P, P, C.POINTER(DynParams), C.c_int32, C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32), P]),
    "mj_plan_set_tma": (C.c_int32, [P, C.c_int32]),
    "mj_plan_set_fused": (C.c_int32, [P, C.c_int32]),
    "mj_plan_set_option": (C.c_int32, [P, C.c_int32, C.c_int32]),
    "mj_plan_check_status": (C.c_int32, [P]),
    "mj_plan_selftest_timeout": (C.c_int32, [P, C.c_uint32, P]),
    "mj_plan_set_bfield": (C.c_int32, [P, P]),
    "mj_plan_set_bfield_device": (C.c_int32, [P, P, P]),
    "mj_state_create": (C.c_int32, [P, C.POINTER(P)]),
    "mj_state_destroy": (C.c_int32, [P]),
    "mj_state_upload": (C.c_int32, [P, P, P]),
    "mj_state_download": (C.c_int32, [P, P, P]),
    "mj_state_device_ptr": (C.c_int32, [P, C.POINTER(P)]),
    "mj_field": (C.c_int32, [P, P, P, P, P]),
    "mj_field_dev": (C.c_int32, [P, P, P, P, P]),
    "mj_energy": (C.c_int32, [P, P, DP]),
    "mj_field_host": (C.c_int32, [P, P, P, P]),
    "mj_energy_noalloc": (C.c_int32, [P, P, P, P]),
    "mj_step": (C.c_int32, [P, P, C.POINTER(DynParams), C.c_int32, P, P]),
    "mj_step_dev": (C.c_int32, [P, P, C.POINTER(DynParams), C.c_int32, P, P]),
    "mj_step_host": (C.c_int32, [P, P, C.POINTER(DynParams), C.c_int32, P]),
    "mj_graph_run": (C.c_int32, [P, P, C.POINTER(DynParams), C.c_int32, C.c_int32, P, P]),
    "mj_profile_enable": (C.c_int32, [P, C.c_int32]),
    "mj_profile_read": (C.c_int32, [P, C.c_int32, P, P, P, C.POINTER(C.c_int32)]),
    "mj_measure_temperature": (C.c_int32, [P, P, DP]),
    "mj_philox_normals": (C.c_int32, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_int64, P, P]),
    "mj_minimize": (C.c_int32, [P, P, C.POINTER(MinParams), C.c_int64, C.POINTER(C.c_int64),
                                C.POINTER(C.c_double), P]),
    "mj_minimize_infdamp": (C.c_int32, [P, P, C.POINTER(MinParams), C.c_int64, C.POINTER(C.c_int64),
                                        C.POINTER(C.c_double), P, P]),
    "mj_mc_sweeps": (C.c_int32, [P, P, C.POINTER(McParams), C.c_int32, P, P, C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int32), P]),
    "mj_plan_nterms": (C.c_int32, [P, C.POINTER(C.c_int32)]),
    "mj_plan_set_terms": (C.c_int32, [P, P]),
    "mj_field_vjp": (C.c_int32, [P, P, P, P, P, P, P]),
    "mj_adjoint_create": (C.c_int32, [P, C.c_int32, C.c_int32, C.POINTER(P)]),
    "mj_adjoint_destroy": (C.c_int32, [P]),
    "mj_adjoint_forward": (C.c_int32, [P, C.POINTER(DynParams), P, P, P]),
    "mj_adjoint_backward": (C.c_int32, [P, P, P, P, P, P]),
    "mj_batch_create": (C.c_int32, [C.POINTER(LatticeDesc), C.POINTER(HamiltonianDesc), C.c_int32, P, P, P,
                                    C.c_int32, C.POINTER(P)]),
    "mj_batch_destroy": (C.c_int32, [P]),
    "mj_batch_nsites": (C.c_int32, [P, C.POINTER(C.c_int64), P]),
    "mj_batch_device_ptr": (C.c_int32, [P, C.POINTER(P)]),
    "mj_batch_upload": (C.c_int32, [P, P, P]),
    "mj_batch_download": (C.c_int32, [P, P, P]),
    "mj_batch_step": (C.c_int32, [P, C.POINTER(DynParams), C.c_int32, C.c_int32, P, P]),
    "mj_batch_graph_run": (C.c_int32, [P, C.POINTER(DynParams), C.c_int32, C.c_int32, C.c_int32, P, P]),
    "mj_batch_energies": (C.c_int32, [P, P]),
    "mj_batch_temperatures": (C.c_int32, [P, P, P]),
    "mj_batch_field": (C.c_int32, [P, P, P, C.c_int32, P]),
    "mj_batch_gneb_tangent": (C.c_int32, [P, P, C.c_int32, P, P]),
    "mj_batch_gneb_path": (C.c_int32, [P, P, P, P, P, P, P, P]),
    "mj_gneb_path": (C.c_int32, [P, P, C.c_int32, P, P, P, P, P, P, P, P]),
    "mj_batch_set_config": (C.c_int32, [P, C.c_int32, C.c_int32]),
    "mj_batch_autotune": (C.c_int32, [P, C.POINTER(DynParams), C.c_int32, C.POINTER(C.c_int32),
                                      C.POINTER(C.c_int32), P]),
    "mj_batch_mc": (C.c_int32, [P, C.POINTER(McParams), C.c_int32, C.c_int32, C.c_int32, P, P, P,
                                C.POINTER(C.c_int32), P]),
    "mj_batch_mc_reset": (C.c_int32, [P, C.c_double]),
    "mj_batch_mc_state": (C.c_int32, [P, P, P, P]),
}


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python matjes_b200/build.py` "
            "(the CUDA library is required; there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int) -> None:
    if status != MJ_OK:
        raise MatjesError(status, lib.mj_last_error().decode())


def profile_read(plan, cap: int = 32) -> dict:
    """{kernel name: (total ms, launches)} recorded since mj_profile_enable."""
    import numpy as np

    names = C.create_string_buffer(32 * cap)
    tot = np.zeros(cap)
    cnt = np.zeros(cap, np.int64)
    n = C.c_int32()
    check(lib.mj_profile_read(plan, cap, C.addressof(names), tot.ctypes.data, cnt.ctypes.data, C.byref(n)))
    out = {}
    for i in range(min(n.value, cap)):
        nm = names.raw[32 * i:32 * i + 32].split(b"\0")[0].decode()
        out[nm] = (float(tot[i]), int(cnt[i]))
    return out


def ptr(arr) -> int:
    """Address of a numpy array or torch tensor (None -> NULL)."""
    if arr is None:
        return None
    if hasattr(arr, "data_ptr"):
        return arr.data_ptr()
    return arr.ctypes.data
