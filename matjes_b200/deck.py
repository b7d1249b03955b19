"""Lattice + Hamiltonian description in the vocabulary of a Matjes input deck.

A ``Deck`` carries what the reference reads from its ``input`` file for this
path (paths relative to Matjes src/):

* ``Nsize``, ``Periodic_log``, ``alat``/``lattice`` -> ``L``, ``periodic``,
  ``areal`` (rows = lattice vectors in nm; IO-input/rw_lattice.f90:28-80)
* ``atomtypes``/``atoms`` -> ``atoms`` = [(fractional position, type, moment)]
  (IO-input/rw_cell.f90:5-31)
* ``magnetic_J t1 t2 shell J`` -> ``J`` (Energy/exchange_Heisenberg_J.f90:18)
* ``magnetic_D t1 t2 mediator shell D`` -> ``D`` (Energy/exchange_Heisenberg_D.f90:17)
* ``magnetic_anisotropy type ex ey ez K`` -> ``K`` (Energy/anisotropy_heisenberg.f90)
* ``H_ext`` -> ``B_ext`` (Energy/zeeman.f90:21)
* ``mag_dip_use``/``mag_dip_period_cut`` -> ``dip``/``dip_cut`` (Energy/dipolar_magnetic.f90:43-52)
* ``c_H_J``, ``c_H_D``, ``c_H_ani``, ``c_zeeman`` prefactors
  (IO-input/input_H_types.f90:69-140: -1, -1, +1, -1).

Energies in eV (input J = 1 meV is ``1e-3``), fields in Tesla, lengths in nm.
An easy axis needs a negative anisotropy input (c_H_ani = +1).  The
precession rate is mu_B mu_s B / hbar, so gamma = 0.176 rad/(ps T) means
mu_s = 2 mu_B.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

Vec3 = Tuple[float, float, float]


@dataclass
class Deck:
    L: Tuple[int, int, int]
    periodic: Tuple[int, int, int]
    areal: np.ndarray
    atoms: List[Tuple[Vec3, int, float]]
    J: List[Tuple[int, int, int, float]] = field(default_factory=list)
    D: List[Tuple[int, int, int, int, float]] = field(default_factory=list)
    K: List[Tuple[int, Vec3, float]] = field(default_factory=list)
    B_ext: Vec3 = (0.0, 0.0, 0.0)
    zeeman_on: bool = False
    dip: int = 0  # FFT dipolar term: 0 off, 1 the reference's grid rule, 2 zero-padded to 2 L on every axis
    dip_cut: Tuple[int, int, int] = (1, 1, 1)
    c_H_J: float = -1.0
    c_H_D: float = -1.0
    c_H_ani: float = 1.0
    c_zeeman: float = -1.0

    # ------------------------------------------------------------------
    @property
    def ncell(self) -> int:
        return int(self.L[0] * self.L[1] * self.L[2])

    @property
    def nmag(self) -> int:
        return sum(1 for a in self.atoms if a[2] > 0)

    @property
    def nsites(self) -> int:
        return self.ncell * self.nmag

    def positions(self) -> np.ndarray:
        """Site positions (nm), shape (N, 3), site = cell*Nmag + imag."""
        Lx, Ly, Lz = self.L
        z, y, x = np.meshgrid(np.arange(Lz), np.arange(Ly), np.arange(Lx), indexing="ij")
        cells = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(float) @ self.areal
        mags = [np.asarray(a[0], float) @ self.areal for a in self.atoms if a[2] > 0]
        return (cells[:, None, :] + np.asarray(mags)[None, :, :]).reshape(-1, 3)

    # ------------------------------------------------------------------
    def c_structs(self):
        """(LatticeDesc, HamiltonianDesc, keep-alive arrays) for the C ABI."""
        # imported here, not at module level: the deck itself needs no CUDA
        # library (a CPU-only consumer can load this file on its own)
        from . import _abi

        lat = _abi.LatticeDesc()
        for d in range(3):
            lat.L[d] = int(self.L[d])
            lat.periodic[d] = int(bool(self.periodic[d]))
            for k in range(3):
                lat.areal[d][k] = float(self.areal[d][k])
        if len(self.atoms) > _abi.MJ_MAX_ATOMS:
            raise ValueError("too many atoms in the cell")
        lat.natom = len(self.atoms)
        for a, (frac, t, mom) in enumerate(self.atoms):
            for k in range(3):
                lat.frac[a][k] = float(frac[k])
            lat.attype[a] = int(t)
            lat.moment[a] = float(mom)
        J = (_abi.ExchangeTerm * max(1, len(self.J)))(*[_abi.ExchangeTerm(t1, t2, s, v) for t1, t2, s, v in self.J])
        D = (_abi.DmiTerm * max(1, len(self.D)))(*[_abi.DmiTerm(t1, t2, tm, s, v) for t1, t2, tm, s, v in self.D])
        Ks = []
        for t, ax, v in self.K:
            a = _abi.AnisoTerm()
            a.type = int(t)
            for k in range(3):
                a.axis[k] = float(ax[k])
            a.value = float(v)
            Ks.append(a)
        K = (_abi.AnisoTerm * max(1, len(Ks)))(*Ks)
        h = _abi.HamiltonianDesc()
        h.nJ, h.J = len(self.J), C.cast(J, C.POINTER(_abi.ExchangeTerm))
        h.nD, h.D = len(self.D), C.cast(D, C.POINTER(_abi.DmiTerm))
        h.nK, h.K = len(self.K), C.cast(K, C.POINTER(_abi.AnisoTerm))
        h.c_H_J, h.c_H_D, h.c_H_ani, h.c_zeeman = self.c_H_J, self.c_H_D, self.c_H_ani, self.c_zeeman
        for k in range(3):
            h.B_ext[k] = float(self.B_ext[k])
            h.dip_period_cut[k] = int(self.dip_cut[k])
        h.zeeman_on = int(bool(self.zeeman_on))
        h.dip_on = int(self.dip)
        return lat, h, (J, D, K)


# ----------------------------------------------------------------------
# lattices
SQRT3 = float(np.sqrt(3.0))


def square_areal(a: float = 1.0, c: float = 1.0) -> np.ndarray:
    return np.array([[a, 0.0, 0.0], [0.0, a, 0.0], [0.0, 0.0, c]])


def triangular_areal(a: float = 1.0, c: float = 1.0) -> np.ndarray:
    """a1 = (1/2, -sqrt3/2, 0), a2 = (1/2, sqrt3/2, 0): the triangular cell of the
    reference's example deck (inputs/input)."""
    return np.array([[0.5 * a, -0.5 * SQRT3 * a, 0.0], [0.5 * a, 0.5 * SQRT3 * a, 0.0], [0.0, 0.0, c]])


def square_film(L, Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.5, mu_s=2.0, periodic=(1, 1, 0), a=1.0,
                med_z=-0.5, dip=False) -> Deck:
    """Square (2D) or simple-cubic (L[2] > 1) lattice, one magnetic atom per
    cell, interfacial DMI from a non-magnetic mediator below the plaquette
    centre (d = z x r_ij on the in-plane bonds)."""
    atoms = [((0.0, 0.0, 0.0), 1, mu_s), ((0.5, 0.5, med_z), 2, 0.0)]
    deck = Deck(L=tuple(L), periodic=tuple(periodic), areal=square_areal(a, a), atoms=atoms,
                J=[(1, 1, 1, Jv)] if Jv else [], D=[(1, 1, 2, 1, Dv)] if Dv else [],
                K=[(1, (0.0, 0.0, 1.0), Kv)] if Kv else [], B_ext=(0.0, 0.0, Bz), dip=dip)
    return deck


def triangular(L, J=(1.0e-3, -0.1e-3, -0.05e-3), Dv=0.2e-3, Kv=-0.05e-3, Bz=1.0, mu_s=2.0) -> Deck:
    """Triangular monolayer with exchange shells J1..Jn and an interfacial D1
    from mediators at both hollow sites, so that d lies in-plane, normal to
    the bond."""
    atoms = [((0.0, 0.0, 0.0), 1, mu_s), ((1.0 / 3.0, 2.0 / 3.0, -0.5), 2, 0.0), ((2.0 / 3.0, 1.0 / 3.0, -0.5), 2, 0.0)]
    Js = [(1, 1, s + 1, v) for s, v in enumerate(J) if v]
    return Deck(L=(L[0], L[1], 1), periodic=(1, 1, 0), areal=triangular_areal(), atoms=atoms, J=Js,
                D=[(1, 1, 2, 1, Dv)] if Dv else [], K=[(1, (0.0, 0.0, 1.0), Kv)] if Kv else [],
                B_ext=(0.0, 0.0, Bz))


# ----------------------------------------------------------------------
# initial states (host AoS, (N, 3))
def random_sphere(n: int, seed: int) -> np.ndarray:
    """Uniform on the unit sphere (z ~ U(-1,1), phi ~ U(0, 2 pi))."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    s = np.sqrt(1.0 - z * z)
    m = np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)
    return m / np.linalg.norm(m, axis=1, keepdims=True)


def reversed_disks(deck: Deck, ndisk: int, radius: float, seed: int) -> np.ndarray:
    """Ferromagnet along +z with `ndisk` disks (radius in lattice spacings,
    periodic minimum image) reversed to -z; centres drawn from `seed`."""
    Lx, Ly, _ = deck.L
    rng = np.random.default_rng(seed)
    cx = rng.integers(0, Lx, ndisk)
    cy = rng.integers(0, Ly, ndisk)
    a1, a2 = deck.areal[0, :2], deck.areal[1, :2]
    flip = np.zeros((Ly, Lx), bool)
    # cell offsets whose distance can be within the radius: |r| >= s_min |(dx, dy)|
    s_min = np.linalg.svd(np.stack([a1, a2]), compute_uv=False).min()
    B = int(np.ceil(radius / s_min)) + 1
    if 2 * B + 2 <= min(Lx, Ly):
        # the disk's bounding box only (its offsets are the minimum images)
        dy, dx = np.meshgrid(np.arange(-B, B + 1), np.arange(-B, B + 1), indexing="ij")
        r = dx[..., None] * a1 + dy[..., None] * a2
        inside = (r ** 2).sum(-1) <= radius * radius + 1e-9
        ox, oy = dx[inside], dy[inside]
        for i in range(ndisk):
            flip[(cy[i] + oy) % Ly, (cx[i] + ox) % Lx] = True
    else:
        y, x = np.meshgrid(np.arange(Ly), np.arange(Lx), indexing="ij")
        for i in range(ndisk):
            dx = (x - cx[i] + Lx // 2) % Lx - Lx // 2
            dy = (y - cy[i] + Ly // 2) % Ly - Ly // 2
            r = dx[..., None] * a1 + dy[..., None] * a2
            flip |= (r ** 2).sum(-1) <= radius * radius + 1e-9
    m = np.zeros((Ly * Lx, 3))
    m[:, 2] = np.where(flip.ravel(), -1.0, 1.0)
    return np.tile(m, (deck.L[2], 1))


# ----------------------------------------------------------------------
# the synthetic workloads (shapes, couplings and seeds of the benchmark configurations)
def workload(name: str, scale: int = 1) -> dict:
    """Return {deck, m0, dyn} for a named workload.  `scale` divides lattice
    sides for small parity runs (e.g. scale=16 turns 1024^2 into 64^2)."""
    if name == "square64_sib":
        L = 64 // scale if scale > 1 else 64
        deck = square_film((L, L, 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.5)
        return dict(deck=deck, m0=random_sphere(deck.nsites, 0),
                    dyn=dict(integrator="sib", timestep=0.1, alpha=0.3, temperature=0.0, steps=1000))
    if name == "triangular1024_thermal":
        L = 1024 // scale
        deck = triangular((L, L))
        return dict(deck=deck, m0=reversed_disks(deck, 20, 8.0, 1),
                    dyn=dict(integrator="sib", timestep=0.1, alpha=0.1, temperature=10.0, noise="philox", seed=1,
                             steps=2000))
    if name == "triangular4096_thermal":
        # the same couplings and dynamics at 4096^2 (16.8 M sites, 403 MB per field:
        # every pass streams from HBM), disks at the 1024^2 density
        L = 4096 // scale
        deck = triangular((L, L))
        return dict(deck=deck, m0=reversed_disks(deck, max(1, 20 * (L // 1024) ** 2), 8.0, 1),
                    dyn=dict(integrator="sib", timestep=0.1, alpha=0.1, temperature=10.0, noise="philox", seed=1,
                             steps=2000))
    if name == "square256_adjoint":
        # parameters J, D, K (global) and a per-site Bz = 0.5 + N(0, 0.05) T (seed 3);
        # the target state comes from J, D, K = 1.1, 0.35, -0.08 meV and
        # Bz = 0.5 + 0.2 sin(2 pi x / L) T from the same initial state
        L = 256 // scale
        deck = square_film((L, L, 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.5)
        rng = np.random.default_rng(3)
        bz = 0.5 + 0.05 * rng.standard_normal(deck.nsites)
        x = np.arange(deck.nsites) % L
        bz_target = 0.5 + 0.2 * np.sin(2.0 * np.pi * x / L)
        return dict(deck=deck, m0=random_sphere(deck.nsites, 3),
                    bfield=np.stack([np.zeros_like(bz), np.zeros_like(bz), bz], axis=1),
                    target_terms=np.array([1.1e-3, 0.35e-3, -0.08e-3]),
                    target_bfield=np.stack([np.zeros_like(bz), np.zeros_like(bz), bz_target], axis=1),
                    dyn=dict(integrator="sib", timestep=0.1, alpha=0.2, temperature=0.0, steps=500,
                             checkpoint_every=50))
    if name == "film128x16_dipolar":
        L = 128 // scale
        Lz = max(2, 16 // scale)
        deck = square_film((L, L, Lz), Jv=1e-3, Dv=0.15e-3, Kv=-0.02e-3, Bz=0.2, a=0.25, med_z=-0.3, dip=True)
        return dict(deck=deck, m0=random_sphere(deck.nsites, 4),
                    dyn=dict(integrator="sib", timestep=0.1, alpha=0.1, temperature=5.0, noise="philox", seed=4,
                             steps=2000))
    if name == "square_replicas256":
        # 256 square replicas, sides drawn from {32..256} (seed 2), Bz ~ U(0, 2) T,
        # temperatures geometric 1 -> 50 K; `scale` divides the sides and the count
        rng = np.random.default_rng(2)
        nrep = max(4, 256 // scale)
        sides = np.array([32, 48, 64, 96, 128, 192, 256])
        Ls = rng.choice(sides, size=256)[:nrep] // scale
        Ls = np.maximum(Ls, 8)
        Bz = rng.uniform(0.0, 2.0, size=256)[:nrep]
        T = 1.0 * (50.0 / 1.0) ** (np.arange(nrep) / max(1, nrep - 1))
        cell = square_film((8, 8, 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.0)
        sizes = np.stack([Ls, Ls], axis=1).astype(np.int32)
        B = np.zeros((nrep, 3))
        B[:, 2] = Bz
        ntot = int((Ls.astype(np.int64) ** 2).sum())
        return dict(cell=cell, sizes=sizes, B_ext=B, temperature=T, m0=random_sphere(ntot, 2),
                    dyn=dict(integrator="sib", timestep=0.1, alpha=0.5, noise="philox", seed=2, steps=5000,
                             swap_every=100))
    raise KeyError(name)
