"""ctypes wrapper of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: what the tests compare the CUDA path against.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference legs may use
it; the product (matjes_b200) never imports it.  See matjes_oracle.h for the
reference routines it restates and for its pinning status.

Decks are duck-typed: any object with the attributes of matjes_b200.deck.Deck
(L, periodic, areal, atoms, J, D, K, B_ext, zeeman_on, dip, dip_cut, c_H_*).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# ORACLE_NATIVE=1 (set by bench.py's CPU-baseline and reference legs before the
# import) loads the -O3 -march=native build made on this machine instead
NATIVE = os.environ.get("ORACLE_NATIVE") == "1"
LIB = os.path.join(HERE, "liboracle_native.so" if NATIVE else "liboracle.so")
MAXAT = 16
MAXTERM = 32
KB = 0.000086173324
MUB = 0.0000578838180661
HBAR = 0.658211928


def build() -> str:
    # the native build is always remade: a copy made on another machine may
    # use instructions this one lacks
    subprocess.run(["make", "-s", "-C", HERE] + (["-B"] if NATIVE else []) + [os.path.basename(LIB)], check=True)
    return LIB


class _Lat(C.Structure):
    _fields_ = [("L", C.c_int * 3), ("periodic", C.c_int * 3), ("areal", (C.c_double * 3) * 3), ("natom", C.c_int),
                ("frac", (C.c_double * 3) * MAXAT), ("attype", C.c_int * MAXAT), ("moment", C.c_double * MAXAT)]


class _J(C.Structure):
    _fields_ = [("t1", C.c_int), ("t2", C.c_int), ("shell", C.c_int), ("J", C.c_double)]


class _D(C.Structure):
    _fields_ = [("t1", C.c_int), ("t2", C.c_int), ("tmed", C.c_int), ("shell", C.c_int), ("D", C.c_double)]


class _K(C.Structure):
    _fields_ = [("type", C.c_int), ("axis", C.c_double * 3), ("K", C.c_double)]


class _Input(C.Structure):
    _fields_ = [("lat", _Lat), ("nJ", C.c_int), ("J", _J * MAXTERM), ("nD", C.c_int), ("D", _D * MAXTERM),
                ("nK", C.c_int), ("K", _K * MAXTERM), ("c_H_J", C.c_double), ("c_H_D", C.c_double),
                ("c_H_ani", C.c_double), ("c_zeeman", C.c_double), ("B_ext", C.c_double * 3), ("zeeman_on", C.c_int),
                ("dip_on", C.c_int), ("dip_period_cut", C.c_int * 3)]


class _Dyn(C.Structure):
    _fields_ = [("integrator", C.c_int), ("timestep", C.c_double), ("alpha", C.c_double),
                ("temperature", C.c_double), ("noise", C.c_int), ("seed", C.c_uint64), ("stream", C.c_uint32),
                ("step0", C.c_uint32), ("inject", C.c_void_p), ("inject_nbuf", C.c_int),
                ("energy_before", C.c_int)]


INTEGRATORS = {"euler": 1, "heun": 2, "heun_matjes": 2, "sib": 3}
NOISES = {"off": 0, "philox": 1, "inject": 2}


def _lib():
    if NATIVE or not os.path.exists(LIB):
        build()  # the native build is made for (and on) the machine that runs it
    lib = C.CDLL(LIB)
    P, DP = C.c_void_p, C.POINTER(C.c_double)
    lib.orc_input_defaults.argtypes = [C.POINTER(_Input)]
    lib.orc_model_build.argtypes = [C.POINTER(_Input), C.POINTER(P)]
    lib.orc_model_build.restype = C.c_int
    lib.orc_model_free.argtypes = [P]
    lib.orc_nsites.argtypes = [P]
    lib.orc_nsites.restype = C.c_int64
    lib.orc_mm_nnz.argtypes = [P]
    lib.orc_mm_nnz.restype = C.c_int64
    lib.orc_mm_coo.argtypes = [P, C.c_int64, P, P, P]
    lib.orc_set_bfield.argtypes = [P, P]
    lib.orc_dip_nrep.argtypes = [P, C.c_int * 3]
    lib.orc_field.argtypes = [P, P, P, P]
    lib.orc_field_terms.argtypes = [P, P, P, P, P]
    lib.orc_energy.argtypes = [P, P]
    lib.orc_energy.restype = C.c_double
    lib.orc_dipolar_explicit_field.argtypes = [P, P, P]
    lib.orc_philox_normals.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_int64, C.c_int64, P]
    lib.orc_philox4x32.argtypes = [P, P, P]
    lib.orc_tab_eval.argtypes = [P, C.c_int64, P, P, P]
    lib.orc_run.argtypes = [P, C.POINTER(_Dyn), P, C.c_int, P]
    lib.orc_run.restype = C.c_int
    lib.orc_llg_torque.argtypes = [P, C.c_double, P, P, C.c_int64]
    return lib


lib = _lib()


def _p(a):
    return None if a is None else a.ctypes.data


class Model:
    """The reference Hamiltonian of a deck, assembled as the reference does."""

    def __init__(self, deck):
        inp = _Input()
        lib.orc_input_defaults(C.byref(inp))
        for d in range(3):
            inp.lat.L[d] = int(deck.L[d])
            inp.lat.periodic[d] = int(bool(deck.periodic[d]))
            for k in range(3):
                inp.lat.areal[d][k] = float(deck.areal[d][k])
        inp.lat.natom = len(deck.atoms)
        for a, (frac, t, mom) in enumerate(deck.atoms):
            for k in range(3):
                inp.lat.frac[a][k] = float(frac[k])
            inp.lat.attype[a] = int(t)
            inp.lat.moment[a] = float(mom)
        inp.nJ = len(deck.J)
        for i, (t1, t2, s, v) in enumerate(deck.J):
            inp.J[i] = _J(t1, t2, s, v)
        inp.nD = len(deck.D)
        for i, (t1, t2, tm, s, v) in enumerate(deck.D):
            inp.D[i] = _D(t1, t2, tm, s, v)
        inp.nK = len(deck.K)
        for i, (t, ax, v) in enumerate(deck.K):
            inp.K[i].type = t
            for k in range(3):
                inp.K[i].axis[k] = ax[k]
            inp.K[i].K = v
        inp.c_H_J, inp.c_H_D, inp.c_H_ani, inp.c_zeeman = deck.c_H_J, deck.c_H_D, deck.c_H_ani, deck.c_zeeman
        for k in range(3):
            inp.B_ext[k] = float(deck.B_ext[k])
            inp.dip_period_cut[k] = int(deck.dip_cut[k])
        inp.zeeman_on = int(bool(deck.zeeman_on))
        inp.dip_on = int(deck.dip)
        h = C.c_void_p()
        rc = lib.orc_model_build(C.byref(inp), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"oracle model build failed ({rc})")
        self.h = h
        self.N = int(lib.orc_nsites(h))

    def __del__(self):
        # at interpreter exit the module globals (lib) may already be gone
        if getattr(self, "h", None) and lib is not None:
            lib.orc_model_free(self.h)
            self.h = None

    def set_bfield(self, b_cell):
        self._b = None if b_cell is None else np.ascontiguousarray(b_cell, np.float64)
        lib.orc_set_bfield(self.h, _p(self._b))

    def field(self, m):
        m = np.ascontiguousarray(m, np.float64)
        B = np.empty_like(m)
        e = np.empty(self.N)
        lib.orc_field(self.h, _p(m), _p(B), _p(e))
        return B, e

    def field_terms(self, m):
        m = np.ascontiguousarray(m, np.float64)
        out = [np.empty_like(m) for _ in range(3)]
        lib.orc_field_terms(self.h, _p(m), *[_p(o) for o in out])
        return out

    def energy(self, m) -> float:
        return float(lib.orc_energy(self.h, _p(np.ascontiguousarray(m, np.float64))))

    def dip_direct(self, direct: bool = True) -> None:
        """Dipolar convolution by the direct circular sum (True) or, on
        power-of-two grids, by the oracle's own FFT (False, the default)."""
        lib.orc_dip_direct.argtypes = [C.c_void_p, C.c_int]
        lib.orc_dip_direct(self.h, int(bool(direct)))

    def dipolar_explicit(self, m):
        m = np.ascontiguousarray(m, np.float64)
        B = np.empty_like(m)
        lib.orc_dipolar_explicit_field(self.h, _p(m), _p(B))
        return B

    def nrep(self):
        a = (C.c_int * 3)()
        lib.orc_dip_nrep(self.h, a)
        return tuple(a)

    def coo(self):
        n = int(lib.orc_mm_nnz(self.h))
        r = np.empty(n, np.int64)
        c = np.empty(n, np.int64)
        v = np.empty(n)
        lib.orc_mm_coo(self.h, n, _p(r), _p(c), _p(v))
        return r, c, v

    def run(self, m, nsteps, integrator="sib", timestep=0.1, alpha=0.1, temperature=0.0, noise="off", seed=0,
            stream=0, step0=0, inject=None, energies=False, energy_before=False, **_ignored):
        """Advance m (N,3) in place; inject is a host array [nbuf][3][N].  With
        `energies`, returns the energy after each step (an extra field pass per
        step), or with `energy_before` the energy of the state each step starts
        from, summed in the step's first field pass."""
        assert m.dtype == np.float64 and m.flags.c_contiguous
        d = _Dyn()
        d.integrator = INTEGRATORS[integrator]
        d.timestep, d.alpha, d.temperature = timestep, alpha, temperature
        d.noise = NOISES[noise]
        d.seed, d.stream, d.step0 = seed, stream, step0
        d.energy_before = int(bool(energy_before))
        keep = None
        if inject is not None:
            keep = np.ascontiguousarray(inject, np.float64)
            d.inject = keep.ctypes.data
            d.inject_nbuf = keep.shape[0]
        E = np.empty(nsteps) if energies else None
        rc = lib.orc_run(self.h, C.byref(d), _p(m), int(nsteps), _p(E))
        if rc != 0:
            raise RuntimeError("oracle run failed")
        return E


def _minimize_bind():
    lib.orc_minimize_vpo.restype = C.c_int
    lib.orc_minimize_vpo.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int64,
                                     C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    lib.orc_minimize_infdamp.restype = C.c_int
    lib.orc_minimize_infdamp.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_int64, C.c_void_p,
                                         C.POINTER(C.c_int64), C.POINTER(C.c_double)]


def minimize_vpo(model, m, dt, mass, conv_torque, niter):
    """solvers/minimize.F90:57-166 on m (N,3) in place; returns (iterations, max torque)."""
    _minimize_bind()
    it, mt = C.c_int64(), C.c_double()
    rc = lib.orc_minimize_vpo(model.h, _p(m), dt, mass, conv_torque, int(niter), C.byref(it), C.byref(mt))
    if rc != 0:
        raise RuntimeError("oracle minimisation failed")
    return it.value, mt.value


def minimize_infdamp(model, m, conv_torque, niter, colors=(1, 1, 1)):
    """solvers/minimize.F90:169-258 on m (N,3) in place, in site order (colors 1 1 1)
    or colour by colour; returns (iterations, max torque)."""
    _minimize_bind()
    c = np.ascontiguousarray(colors, np.int32)
    it, mt = C.c_int64(), C.c_double()
    rc = lib.orc_minimize_infdamp(model.h, _p(m), conv_torque, int(niter), c.ctypes.data, C.byref(it), C.byref(mt))
    if rc != 0:
        raise RuntimeError(f"oracle infinite-damping minimisation failed ({rc})")
    return it.value, mt.value


class MC(C.Structure):
    """orc_mc: the chain state carried between calls (cone, counts, next sweep)."""
    _fields_ = [("temperature", C.c_double), ("cone", C.c_double), ("proposal", C.c_int),
                ("adapt_cone", C.c_int), ("seed", C.c_uint64), ("stream_id", C.c_uint32),
                ("sweep0", C.c_uint32), ("accepted_total", C.c_int64), ("proposed_total", C.c_int64)]


def _mc_bind():
    lib.orc_mc_sweeps.restype = C.c_int
    lib.orc_mc_sweeps.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(MC), C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                  C.c_void_p, C.POINTER(C.c_int64)]
    lib.orc_mc_random.restype = C.c_int
    lib.orc_mc_random.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(MC), C.c_int, C.c_void_p, C.c_void_p,
                                  C.POINTER(C.c_int64)]


def mc_site_colours(L, colors):
    """Per-site colour (x fastest) of a colouring {q, b, c, 1} (linear, (x + b y +
    c z) mod q) or {cx, cy, cz, 0} (product, x mod cx fastest); and the count."""
    z, y, x = np.meshgrid(np.arange(L[2]), np.arange(L[1]), np.arange(L[0]), indexing="ij")
    a0, a1, a2, form = (int(v) for v in colors)
    if form == 1:
        return np.ascontiguousarray(((x + a1 * y + a2 * z) % a0).ravel(), np.int32), a0
    return np.ascontiguousarray(((x % a0) + a0 * ((y % a1) + a1 * (z % a2))).ravel(), np.int32), a0 * a1 * a2


def mc_sweeps(model, m, st: MC, nsweeps, colors, L):
    """Metropolis sweeps colour by colour on m (N,3) in place (Metropolis-MC/MCstep.f90
    moves in the device's site order, `colors` the device's colouring of the
    lattice of sizes L); returns (E per sweep, summed spins per sweep, accepted)."""
    _mc_bind()
    sc, nc = mc_site_colours(L, colors)
    E, Mg, acc = np.empty(nsweeps), np.empty((nsweeps, 3)), C.c_int64()
    rc = lib.orc_mc_sweeps(model.h, _p(m), C.byref(st), int(nsweeps), sc.ctypes.data, nc, _p(E), _p(Mg),
                           C.byref(acc))
    if rc != 0:
        raise RuntimeError(f"oracle Monte Carlo failed ({rc})")
    return E, Mg, acc.value


def mc_random(model, m, st: MC, nsweeps):
    """Metropolis moves at randomly chosen sites as the reference makes them
    (choose_spin, MCstep), N moves per sweep; returns (tracked E, summed spins, accepted)."""
    _mc_bind()
    E, Mg, acc = np.empty(nsweeps), np.empty((nsweeps, 3)), C.c_int64()
    rc = lib.orc_mc_random(model.h, _p(m), C.byref(st), int(nsweeps), _p(E), _p(Mg), C.byref(acc))
    if rc != 0:
        raise RuntimeError(f"oracle Monte Carlo failed ({rc})")
    return E, Mg, acc.value


def gneb_find_path(model, images, spring=0.5, dt=0.01, mass=1.0, ftol=1e-8, itrmax=10 ** 7, en_zero="I",
                   climb=False, return_ci=False):
    """GNEB find_path on images (nim, N, 3), relaxed in place; returns (rx, ene,
    dene, iterations, max |F|) as en_path.out holds them, and the climbing
    image (0-based, -1 without) when return_ci."""
    lib.orc_gneb_find_path.restype = C.c_int
    lib.orc_gneb_find_path.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_int64, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_int64), C.POINTER(C.c_double), C.POINTER(C.c_int)]
    assert images.dtype == np.float64 and images.flags.c_contiguous and images.ndim == 3
    nim = images.shape[0]
    rx, ene, dene = np.zeros(nim), np.zeros(nim), np.zeros(nim)
    it, fc, ci = C.c_int64(), C.c_double(), C.c_int()
    rc = lib.orc_gneb_find_path(model.h, _p(images), nim, spring, dt, mass, ftol, int(itrmax), ord(en_zero),
                                int(bool(climb)), _p(rx), _p(ene), _p(dene), C.byref(it), C.byref(fc), C.byref(ci))
    if rc != 0:
        raise RuntimeError(f"oracle GNEB failed ({rc})")
    if return_ci:
        return rx, ene, dene, it.value, fc.value, ci.value
    return rx, ene, dene, it.value, fc.value


def set_threads(n: int) -> None:
    """OpenMP threads of the oracle's parallel loops (n <= 0: all processors)."""
    lib.orc_set_threads.argtypes = [C.c_int]
    lib.orc_set_threads(int(n))


def philox_normals(seed, step, stream, site0, n):
    out = np.empty((n, 3))
    lib.orc_philox_normals(seed, step, stream, site0, n, _p(out))
    return out


def philox4x32(ctr, key):
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib.orc_philox4x32(c.ctypes.data, k.ctypes.data, out.ctypes.data)
    return [int(x) for x in out]


def tab_eval(w):
    """(log u, sin 2 pi u, cos 2 pi u) of u = (w + 1/2) 2^-32 for 32-bit words w,
    through the Box-Muller tables."""
    w = np.ascontiguousarray(w, np.uint32)
    lg, s, c = (np.empty(w.size) for _ in range(3))
    lib.orc_tab_eval(w.ctypes.data, w.size, lg.ctypes.data, s.ctypes.data, c.ctypes.data)
    return lg, s, c


def llg_torque(B, alpha, m):
    B = np.ascontiguousarray(B, np.float64)
    m = np.ascontiguousarray(m, np.float64)
    D = np.empty_like(m)
    lib.orc_llg_torque(_p(B), alpha, _p(m), _p(D), m.shape[0])
    return D


def pt_uniform(seed: int, l: int, round_idx: int) -> float:
    """The uniform of the swap test of ladder pair (l, l+1) in round round_idx:
    Philox4x32-10 of counter (l, round, 0x50545357, 2) under key `seed`, the
    53-bit uniform [0, 1) of its first two words."""
    w = philox4x32([l & 0xFFFFFFFF, round_idx & 0xFFFFFFFF, 0x50545357, 2],
                   [seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF])
    k = ((w[0] >> 5) << 26) | (w[1] >> 6)
    return k * (1.0 / 9007199254740992.0)


def pt_round(kT_slot, image, E, sizes, round_idx: int, seed: int):
    """One parallel-tempering round (paratemp-MC/paratemp.f90:84-99, accept
    :105-119): ladder pairs (l, l+1) from l = round % 2 in steps of 2, replicas
    of equal size only; delta = (1/kT_{l+1} - 1/kT_l)(E_{l+1} - E_l), accepted
    if delta > 0 or exp(max(delta, -200)) > u.  Returns the new slot -> replica
    map and the accepted pairs."""
    image = list(image)
    accepted = []
    for l in range(round_idx % 2, len(image) - 1, 2):
        a, b = image[l], image[l + 1]
        if tuple(sizes[a]) != tuple(sizes[b]):
            continue
        delta = (1.0 / kT_slot[l + 1] - 1.0 / kT_slot[l]) * (E[b] - E[a])
        acc = delta > 0.0
        if not acc:
            acc = np.exp(max(delta, -200.0)) > pt_uniform(seed, l, round_idx)
        if acc:
            image[l], image[l + 1] = b, a
            accepted.append(l)
    return image, accepted
