"""Minimum-energy paths by the geodesic nudged elastic band (GNEB/ of the reference).

``GNEBInput`` carries the reference's GNEB input (IO-input/GNEB_io.f90, same
names and defaults).  ``geodesic_path`` builds the initial path
(GNEB/path.f90:100-174), ``find_path`` relaxes it on the device
(GNEB/gneb_utils.f90:19-240 find_path, velocity projection; the images held
as the replicas of a ReplicaBatch, mj_batch_gneb_path, or, for lattices and
terms a batch does not hold, on a plan, mj_gneb_path; with the climbing image
for do_gneb_ci), ``hermite_fit``, ``find_sp`` and ``spline_hermite_val``
interpolate the energy along the path and locate the saddle point
(extrapolation/spline.f90, gneb_utils.f90:242-291), ``saddle_configuration``
interpolates the spins there (find_SP_conf, gneb_utils.f90:305-380),
``write_en`` writes en_path.in / en_path.out / enfit_path.out / ensp_path.out
(GNEB/io-gneb.f90:91-120), ``write_image`` the image-GNEB_<k>.dat files
(io-gneb.f90 write_path), and ``gneb_run`` is GNEB_run (GNEB/gneb.f90:33-120):
path initialisation, the relaxations, the outputs.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np


@dataclass
class GNEBInput:
    """IO-input/GNEB_io.f90 GNEB_input (keyword names in the comments)."""
    nim: int = 10                       # nim
    spring: float = 0.5                 # spring
    dt: float = 1.0e-2                  # vpo_dt
    mass: float = 1.0                   # vpo_mass
    itrmax: int = 2 ** 63 - 1           # mep_itrmax
    mepftol: float = 1.0e-3             # mep_ftol
    mepftol_ci: float = 1.0e-5          # mep_ftol_ci
    every: int = 10                     # meptraj_step
    amp_rnd: float = 0.0                # amp_rnd
    amp_rnd_path: float = 0.0           # amp_rnd_path
    en_zero: str = "N"                  # en_zero: 'I' initial image, 'F' final image, 'N' none
    do_norm_rx: str = "N"               # do_norm_rx
    sample_num: int = 500               # sample_num
    do_gneb: bool = False               # do_gneb_simple
    do_gneb_ci: bool = False            # do_gneb_ci
    momfile_i: str = "momfile_i"        # momfile_i
    momfile_f: str = "momfile_f"        # momfile_f
    restartfile_path: str = "nofile"    # restartfile_path
    initpath: int = -1                  # initpath
    read_path: bool = False             # gnebinit_read_path
    read_outer: bool = True             # gnebinit_read_outer
    min_type: int = 1                   # gnebinit_min_type: 0 none, 1 minimize_infdamp, 2 minimize


@dataclass
class GNEBResult:
    """A relaxed path: images (nim, N, 3); rx, ene, dene as en_path.out holds
    them; iterations and final max |F|; the climbing image (0-based, -1 none)."""
    images: np.ndarray
    rx: np.ndarray
    ene: np.ndarray
    dene: np.ndarray
    iterations: int
    max_force: float
    ci: int = -1


def _calc_ang(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.arctan2(np.linalg.norm(np.cross(a, b), axis=-1), (a * b).sum(-1))


def geodesic_path(m_i: np.ndarray, m_f: np.ndarray, nim: int, amp_rnd: float = 0.0, seed: int = 0) -> np.ndarray:
    """geodesic_path (GNEB/path.f90:100-174): every spin rotated from its initial
    to its final direction in nim - 1 equal steps about their common normal; an
    antiparallel pair rotates about an axis drawn once at random and kept for
    the following sites; then every component of every image, the end images
    included, is moved by amp_rnd * 2 (u - 1), u uniform, and renormalised.
    Returns (nim, N, 3)."""
    rng = np.random.default_rng(seed)
    m_i = np.asarray(m_i, float)
    m_f = np.asarray(m_f, float)
    N = m_i.shape[0]
    eps = np.finfo(float).eps
    path = np.zeros((nim, N, 3))
    ax = np.zeros(3)
    for s in range(N):
        ni, nf = m_i[s], m_f[s]
        angle = float(_calc_ang(ni, nf))
        path[0, s], path[-1, s] = ni, nf
        if angle < eps:
            vec = (nf - ni) / (nim - 1)
            for k in range(1, nim - 1):
                p = ni + k * vec
                path[k, s] = p / np.linalg.norm(p)
            continue
        if abs(angle - math.pi) < eps:
            ax = ax - (ax @ ni) * ni
            while np.linalg.norm(ax) < eps:
                ax = 2.0 * rng.uniform(size=3)
                ax = ax - (ax @ ni) * ni
            ax = ax / np.linalg.norm(ax)
            dtheta = math.pi / (nim - 1)
        else:
            c = np.cross(ni, nf)
            ax = c / np.linalg.norm(c)
            dtheta = angle / (nim - 1)
        for k in range(1, nim - 1):
            th = k * dtheta
            p = ni * math.cos(th) + math.sin(th) * np.cross(ax, ni)
            path[k, s] = p / np.linalg.norm(p)
    if amp_rnd != 0.0:
        for k in range(nim):
            for s in range(N):
                d = path[k, s] + amp_rnd * 2.0 * (rng.uniform(size=3) - 1.0)
                n = np.linalg.norm(d)
                if n > 1e-8:
                    path[k, s] = d / n
    return path


def hermite_fit(rx, ene, dene, nn: int):
    """hermite_fit (extrapolation/spline.f90): the piecewise cubic Hermite
    coefficients c (4, nim) through (rx, ene) with slopes dene, and nn samples
    (x, y, dy/dx) evenly spaced over [rx_0, rx_last]."""
    x = np.asarray(rx, float)
    n = x.shape[0]
    c = np.zeros((4, n))
    c[0] = ene
    c[1] = dene
    for i in range(n - 1):
        dt = x[i + 1] - x[i]
        d1 = (c[0, i + 1] - c[0, i]) / dt
        d3 = c[1, i] + c[1, i + 1] - 2.0 * d1
        c[2, i] = (d1 - c[1, i] - d3) / dt
        c[3, i] = d3 / (dt * dt)
    dx = (x[-1] - x[0]) / (nn - 1)
    xx = x[0] + np.arange(nn) * dx
    yy, dyy = np.empty(nn), np.empty(nn)
    for k in range(nn):
        yy[k], dyy[k] = spline_hermite_val(x, c, xx[k])
    return c, xx, yy, dyy


def spline_hermite_val(rx, c, t: float) -> Tuple[float, float]:
    """spline_hermite_val: value and slope at t (the interval of rvec_bracket)."""
    x = np.asarray(rx, float)
    n = x.shape[0]
    left = n - 2
    for i in range(1, n - 1):
        if t < x[i]:
            left = i - 1
            break
    dt = t - x[left]
    s = c[0, left] + dt * (c[1, left] + dt * (c[2, left] + dt * c[3, left]))
    ds = c[1, left] + dt * (2.0 * c[2, left] + dt * 3.0 * c[3, left])
    return float(s), float(ds)


def find_sp(rx, c) -> Tuple[int, float]:
    """find_SP (GNEB/gneb_utils.f90:242-291): the image of highest energy and,
    from the zero of the cubic's slope on the neighbouring interval, the
    offset of the energy maximum from image imax (0-based)."""
    x = np.asarray(rx, float)
    n = x.shape[0]
    eps = np.finfo(float).eps
    ci = 0
    for i in range(n):
        if c[0, i] > c[0, ci]:
            ci = i
    if abs(c[1, ci]) < eps or (ci == 0 and c[1, ci] < 0.0) or (ci == n - 1 and c[1, ci] > 0.0):
        return ci, 0.0
    imax = ci if c[1, ci] > 0.0 else ci - 1
    dl = x[imax + 1] - x[imax]
    d = c[2, imax] ** 2 - 3.0 * c[3, imax] * c[1, imax]
    if d < 0.0:
        raise ValueError("energy maximum has not been found")
    q = -(c[2, imax] + math.copysign(1.0, c[2, imax]) * math.sqrt(d))
    x1 = q / (c[3, imax] * 3.0)
    x2 = c[1, imax] / q
    if 0.0 < x1 < dl:
        return imax, float(x1)
    if 0.0 < x2 < dl:
        return imax, float(x2)
    raise ValueError("energy maximum has not been found")


class PlanPath:
    """A path of nim images held on the device for one plan (a Hamiltonian):
    image r the SoA block (3, N) of a (nim, 3, N) tensor.  The images' fields
    and energies are the plan's own, so any lattice of one magnetic atom per
    cell and any term a plan holds (the FFT dipolar term, 3D films, ELL
    couplings) reaches the GNEB: mj_gneb_path.  The same calls as a ReplicaBatch holding a path."""

    def __init__(self, ham, images: np.ndarray):
        import torch

        img = np.ascontiguousarray(images, np.float64)
        if img.ndim != 3 or img.shape[2] != 3 or img.shape[0] < 3 or img.shape[1] != ham.N:
            raise ValueError("images are (nim >= 3, plan sites, 3)")
        self.ham = ham
        self.nrep = img.shape[0]
        self.m = torch.tensor(img.transpose(0, 2, 1).copy(), device=f"cuda:{ham.device}")

    def gneb_path(self, spring: float = 0.5, dt: float = 1.0e-2, mass: float = 1.0, ftol: float = 1.0e-3,
                  itrmax: int = 2 ** 62, en_zero: str = "N", climb: bool = False):
        """As ReplicaBatch.gneb_path: (rx, ene, dene, iterations, max |F|,
        climbing image or -1); the path is left relaxed."""
        import ctypes as C

        import torch

        from . import _abi
        from ._abi import check, lib, ptr

        if en_zero not in ("I", "F", "N"):
            raise ValueError("en_zero is 'I', 'F' or 'N'")
        p = _abi.GnebParams(float(spring), float(dt), float(mass), float(ftol), int(itrmax), ord(en_zero),
                            int(bool(climb)))
        rx, ene, dene = np.zeros(self.nrep), np.zeros(self.nrep), np.zeros(self.nrep)
        it, fc, ci = C.c_int64(), C.c_double(), C.c_int32()
        stream = torch.cuda.current_stream(self.m.device).cuda_stream
        check(lib.mj_gneb_path(self.ham.plan, ptr(self.m), self.nrep, C.byref(p), ptr(rx), ptr(ene), ptr(dene),
                               C.byref(it), C.byref(fc), C.byref(ci), stream))
        return rx, ene, dene, int(it.value), float(fc.value), int(ci.value)

    def download(self) -> np.ndarray:
        """The images as (nim * N, 3)."""
        return self.m.cpu().numpy().transpose(0, 2, 1).reshape(-1, 3)


def path_holder(deck, images: np.ndarray, device: int = 0, ham=None):
    """The device holder of a path of deck: the replicas of a ReplicaBatch (the
    fused GNEB field pass) for a single-atom 2D square or triangular lattice
    without the dipolar term, else a PlanPath on the deck's plan (ham, when
    given, is that plan)."""
    from . import Hamiltonian
    from ._abi import MJ_ERR_UNSUPPORTED, MatjesError
    from .batch import ReplicaBatch

    img = np.ascontiguousarray(images, np.float64)
    nim, N = img.shape[0], img.shape[1]
    if deck.nmag == 1 and not deck.dip and deck.L[2] == 1:
        try:
            batch = ReplicaBatch(deck, [deck.L[:2]] * nim, np.tile(np.asarray(deck.B_ext, float), (nim, 1)),
                                 [0.0] * nim, device=device)
        except MatjesError as e:
            if e.status != MJ_ERR_UNSUPPORTED:
                raise
        else:
            batch.upload(img.reshape(nim * N, 3))
            return batch
    return PlanPath(ham if ham is not None else Hamiltonian(deck, device=device), img)


def find_path(deck, images: np.ndarray, inp: GNEBInput = GNEBInput(), device: int = 0,
              climb: bool = False) -> GNEBResult:
    """Relax the path images (nim, N, 3) of deck (its lattice, boundaries,
    couplings, field and dipolar term) on the device: GNEB find_path with the
    end images fixed, tolerance mep_ftol (mep_ftol_ci with climb); the images
    held as replicas or on the deck's plan (path_holder)."""
    img = np.ascontiguousarray(images, np.float64)
    nim, N = img.shape[0], img.shape[1]
    if img.ndim != 3 or img.shape[2] != 3 or nim < 3 or N != deck.nsites:
        raise ValueError("images are (nim >= 3, deck sites, 3)")
    return _relax(path_holder(deck, img, device), nim, N, inp, climb)


def find_path_plan(ham, images: np.ndarray, inp: GNEBInput = GNEBInput(), climb: bool = False) -> GNEBResult:
    """find_path on the plan of a Hamiltonian (a deck's, or an ELL plan from
    COO couplings): images (nim, ham.N, 3)."""
    img = np.ascontiguousarray(images, np.float64)
    return _relax(PlanPath(ham, img), img.shape[0], img.shape[1], inp, climb)


def _relax(batch, nim: int, N: int, inp: GNEBInput, climb: bool, itrmax: Optional[int] = None) -> GNEBResult:
    ftol = inp.mepftol_ci if climb else inp.mepftol
    rx, ene, dene, iters, fchk, ci = batch.gneb_path(inp.spring, inp.dt, inp.mass, ftol,
                                                     inp.itrmax if itrmax is None else itrmax, inp.en_zero, climb)
    return GNEBResult(batch.download().reshape(nim, N, 3), rx, ene, dene, iters, fchk, ci)


def saddle_configuration(m1: np.ndarray, m2: np.ndarray, l1: float, l2: float, lsp: float,
                         seed: int = 0) -> np.ndarray:
    """find_SP_conf (GNEB/gneb_utils.f90:305-380): every spin on the geodesic
    from its image-imax direction m1 to its image-imax+1 direction m2, a
    fraction (lsp - l1) / (l2 - l1) of the way: linear and renormalised for
    parallel spins; about m1 x m2 by that fraction of their angle otherwise; for
    antiparallel spins by that fraction of pi about an axis drawn at random
    (numpy's generator from seed, not the reference's) and kept for the
    following sites.  Returns (N, 3)."""
    rng = np.random.default_rng(seed)
    m1 = np.asarray(m1, float)
    m2 = np.asarray(m2, float)
    eps = np.finfo(float).eps
    frac = (lsp - l1) / (l2 - l1)
    out = np.empty_like(m1)
    ax = np.zeros(3)
    for s in range(m1.shape[0]):
        ni, nf = m1[s], m2[s]
        angle = float(_calc_ang(ni, nf))
        if angle < eps:
            p = ni + (nf - ni) * frac
            out[s] = p / np.linalg.norm(p)
            continue
        if abs(angle - math.pi) < eps:
            ax = ax - (ax @ ni) * ni
            while np.linalg.norm(ax) < eps:
                ax = np.sign(2.0 * rng.uniform(size=3) - 1.0) * (rng.uniform(size=3) + 1.0)
                ax = ax - (ax @ ni) * ni
            ax = ax / np.linalg.norm(ax)
            theta = math.pi * frac
        else:
            c = np.cross(ni, nf)
            ax = c / np.linalg.norm(c)
            theta = angle * frac
        p = ni * math.cos(theta) + math.sin(theta) * np.cross(ax, ni)
        out[s] = p / np.linalg.norm(p)
    return out


def write_image(path: str, m: np.ndarray) -> None:
    """One spin per line, 3(F14.8) then two blanks (IO-utils/io-utils.f90
    dump_config of a 2D array, as image-GNEB_<k>.dat holds the images)."""
    m = np.asarray(m, float).reshape(-1, 3)
    with open(path, "w") as f:
        for row in m:
            f.write("".join(f"{v:14.8f}" for v in row) + "  \n")


def write_path(directory: str, images: np.ndarray) -> None:
    """write_path (GNEB/io-gneb.f90:46-57): image-GNEB_<k>.dat, k = 1 .. nim."""
    for k, m in enumerate(images, start=1):
        write_image(os.path.join(directory, f"image-GNEB_{k}.dat"), m)


def write_en(path: str, x, y, dy, x0: Optional[float] = None, do_norm_rx: str = "Y") -> None:
    """write_en (GNEB/io-gneb.f90:91-120): rows x / x0 (do_norm_rx 'Y', x0
    given) or x ('N'), y, dy in 3(E20.12E3, 3X)."""
    from .reference_io import fortran_e

    if do_norm_rx not in ("Y", "N"):
        raise ValueError("Invalid value for do_norm_rx!")
    norm = float(x0) if (do_norm_rx == "Y" and x0 is not None) else 1.0
    with open(path, "w") as f:
        for a, b, d in zip(x, y, dy):
            f.write("".join(fortran_e(v, 20, 12, 3) + "   " for v in (a / norm, b, d)) + "\n")


def saddle_point(rx, ene, dene, sample_num: int = 500):
    """The interpolated energy profile and its maximum, as GNEB_run writes them:
    (x, y, dy) samples (enfit_path.out) and (rx0, E0, dE0) (ensp_path.out)."""
    c, xx, yy, dyy = hermite_fit(rx, ene, dene, sample_num)
    imax, drx0 = find_sp(rx, c)
    rx0 = float(np.asarray(rx)[imax] + drx0)
    e0, de0 = spline_hermite_val(rx, c, rx0)
    return (xx, yy, dyy), (rx0, e0, de0)


def gneb_run(deck, inp: GNEBInput, m_first: Optional[np.ndarray] = None, m_last: Optional[np.ndarray] = None,
             path: Optional[np.ndarray] = None, minimize_input=None, directory: Optional[str] = None,
             device: int = 0, seed: int = 0) -> dict:
    """GNEB_run (GNEB/gneb.f90:33-120) of any deck a plan holds.  Path
    initialisation (GNEB/initialize_path.f90): the given path (read_path), its
    end images replaced by m_first / m_last (read_outer), those minimised
    (min_type 1 minimize_infdamp, 2 minimize, with minimize_input: mass,
    timestep, steps, conv_torque; 0 none), then, unless read_path, the geodesic
    path between them perturbed by amp_rnd_path.  Then find_path (do_gneb,
    mep_ftol) and the climbing-image find_path (do_gneb_ci, mep_ftol_ci), each
    writing en_path.in (the path it starts from); en_path.out, the images, the
    Hermite fit (enfit_path.out), the saddle point (ensp_path.out) and its spins
    (image-GNEB-saddlepoint.dat; the climbing image with do_gneb_ci, else
    saddle_configuration).  Files go to directory when given (the povray files
    of the reference are not written).  Returns the path, rx, ene, dene, the
    saddle point (rx0, E0, dE0) and its spins, and the results of the runs."""
    import torch

    from . import Hamiltonian
    from .hamiltonian import minimize

    nim, N = inp.nim, deck.nsites
    if nim < 3:
        raise ValueError("GNEB needs nim >= 3")
    images = np.zeros((nim, N, 3))
    if inp.read_path:
        if path is None:
            raise ValueError("read_path needs the path")
        images[:] = np.asarray(path, float).reshape(nim, N, 3)
    if inp.read_outer:
        if m_first is None or m_last is None:
            raise ValueError("read_outer needs the initial and final states")
        images[0] = m_first
        images[-1] = m_last

    def out(name):
        return None if directory is None else os.path.join(directory, name)

    if directory is not None:
        write_image(out("SpinSTM_GNEB_ini.dat"), images[0])
        write_image(out("SpinSTM_GNEB_fin.dat"), images[-1])
    if inp.min_type in (1, 2):
        ham = Hamiltonian(deck, device=device)
        mi = minimize_input
        kw = {} if mi is None else dict(timestep=mi.timestep, mass=mi.mass, conv_torque=mi.conv_torque,
                                        max_iter=int(min(mi.steps, 2 ** 62)))
        for k in (0, nim - 1):
            m = torch.tensor(images[k].T.copy(), device=f"cuda:{device}")
            minimize(ham, m, "infdamp" if inp.min_type == 1 else "vpo", **kw)
            images[k] = m.cpu().numpy().T
    elif inp.min_type != 0:
        raise ValueError("UNEXPECTED io_gneb%min_type")
    if not inp.read_path:
        images = geodesic_path(images[0], images[-1], nim, inp.amp_rnd_path, seed)
    if directory is not None:
        write_path(directory, images)
    batch = path_holder(deck, images, device, ham if inp.min_type in (1, 2) else None)
    rx, ene, dene = np.zeros(nim), np.zeros(nim), np.zeros(nim)
    runs = []
    for climb, on in ((False, inp.do_gneb), (True, inp.do_gneb_ci)):
        if not on:
            continue
        start = _relax(batch, nim, N, inp, climb, itrmax=0)
        if directory is not None:
            write_en(out("en_path.in"), start.rx, start.ene, start.dene, start.rx[-1], inp.do_norm_rx)
        r = _relax(batch, nim, N, inp, climb)
        runs.append(r)
        images, rx, ene, dene = r.images, r.rx, r.ene, r.dene
    if directory is not None:
        write_en(out("en_path.out"), rx, ene, dene, rx[-1], inp.do_norm_rx)
        write_path(directory, images)
    c, xx, yy, dyy = hermite_fit(rx, ene, dene, inp.sample_num)
    if directory is not None:
        write_en(out("enfit_path.out"), xx, yy, dyy, rx[-1], inp.do_norm_rx)
    if inp.do_gneb_ci and runs:
        ci = runs[-1].ci
        rx0 = float(rx[ci])
        spinsp = images[ci].copy()
    else:
        imax, drx0 = find_sp(rx, c)
        rx0 = float(rx[imax] + drx0)
        spinsp = images[-1].copy() if imax == nim - 1 else saddle_configuration(
            images[imax], images[imax + 1], rx[imax], rx[imax + 1], rx0, seed)
    e0, de0 = spline_hermite_val(rx, c, rx0)
    if directory is not None:
        write_en(out("ensp_path.out"), [rx0], [e0], [de0], rx[-1], inp.do_norm_rx)
        write_image(out("image-GNEB-saddlepoint.dat"), spinsp)
    return {"images": images, "rx": rx, "ene": ene, "dene": dene, "saddle": (rx0, e0, de0), "saddle_spins": spinsp,
            "runs": runs}
