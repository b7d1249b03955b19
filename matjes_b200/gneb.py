"""Minimum-energy paths by the geodesic nudged elastic band (GNEB/ of the reference).

``GNEBInput`` carries the reference's GNEB input (IO-input/GNEB_io.f90, same
names and defaults).  ``geodesic_path`` builds the initial path
(GNEB/path.f90:100-174), ``find_path`` relaxes it on the device
(GNEB/gneb_utils.f90:19-240 find_path, velocity projection on the images held
as the replicas of a ReplicaBatch: mj_batch_gneb_path), ``hermite_fit``,
``find_sp`` and
``spline_hermite_val`` interpolate the energy along the path and locate the
saddle point (extrapolation/spline.f90, gneb_utils.f90:242-291), ``write_en``
writes en_path.out / enfit_path.out / ensp_path.out (GNEB/io-gneb.f90:83-111).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np

from . import _abi
from ._abi import check, lib, ptr


@dataclass
class GNEBInput:
    """IO-input/GNEB_io.f90 GNEB_input (the path-relaxation part)."""
    nim: int = 10
    spring: float = 0.5
    dt: float = 1.0e-2          # vpo_dt
    mass: float = 1.0           # vpo_mass
    itrmax: int = 2 ** 62       # mep_itrmax
    mepftol: float = 1.0e-3     # mep_ftol
    amp_rnd_path: float = 0.0
    en_zero: str = "N"          # 'I' initial image, 'F' final image, 'N' none
    do_norm_rx: str = "N"
    sample_num: int = 500


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


def find_path(deck, images: np.ndarray, inp: GNEBInput = GNEBInput(), device: int = 0):
    """Relax the path images (nim, N, 3) of the single-atom 2D lattice of deck
    (its L, boundaries, couplings and field) on the device: GNEB find_path with
    the end images fixed.  Returns (relaxed images (nim, N, 3), rx, ene, dene,
    iterations, max |F|); rx / ene / dene as en_path.out holds them."""
    from .batch import ReplicaBatch

    img = np.ascontiguousarray(images, np.float64)
    nim, N = img.shape[0], img.shape[1]
    if img.ndim != 3 or img.shape[2] != 3 or nim < 3 or N != deck.ncell:
        raise ValueError("images are (nim >= 3, deck sites, 3)")
    batch = ReplicaBatch(deck, [deck.L[:2]] * nim, np.tile(np.asarray(deck.B_ext, float), (nim, 1)), [0.0] * nim,
                         device=device)
    batch.upload(img.reshape(nim * N, 3))
    rx, ene, dene, iters, fchk = batch.gneb_path(inp.spring, inp.dt, inp.mass, inp.mepftol, inp.itrmax, inp.en_zero)
    return batch.download().reshape(nim, N, 3), rx, ene, dene, iters, fchk


def write_en(path: str, x, y, dy, x0: Optional[float] = None) -> None:
    """write_en (GNEB/io-gneb.f90:83-111): rows x/x0, y, dy in 3(E20.12E3, 3X)."""
    from .reference_io import fortran_e

    norm = 1.0 if x0 is None else float(x0)
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
