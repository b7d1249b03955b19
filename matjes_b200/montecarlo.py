"""Metropolis Monte Carlo on the device (Metropolis-MC/ of the reference).

``MCInput`` carries the reference's Monte Carlo input (IO-input/MC_io.f90:8-35,
same names and defaults).  ``MetropolisMC`` stands in for ``track_val`` plus
``MCstep`` (Metropolis-MC/track_value.f90, MCstep.f90): it holds the chain
state that persists across temperatures (cone, accepted and proposed counts)
and runs sweeps through ``mj_mc_sweeps``.  ``parallel_tempering_run`` is the
replica-exchange loop of paratemp-MC/parallel_tempering.f90 on a batch of
replicas (``mj_batch_mc``).  ``montecarlo_run`` is the
temperature loop of Metropolis-MC/MonteCarlo.f90:35-162 (relaxation, then
Total_MC_Steps measurements T_auto sweeps apart), ``therm_set`` the averages of
Metropolis-MC/thermo_val.f90:44-77 and ``thermo_print`` the EM.dat rows of
:102-129.

One sweep moves every site once, colour by colour, where the reference moves
N randomly chosen sites (choose_spin); a reference "MC step" count of
T_auto * N moves is T_auto sweeps here.  Topological charge, vortex and
correlation columns are not computed and hold zeros.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _abi
from ._abi import check, lib, ptr
from .hamiltonian import Hamiltonian, _is_torch, _stream

KB = 0.000086173324  # eV / K, fixed-parameters/constant.f90

SAMPLING = {"sphere": _abi.MJ_MC_CONE, "equi": _abi.MJ_MC_CONE, "ising": _abi.MJ_MC_ISING,
            "underrelax": _abi.MJ_MC_UNDERRELAX, "overrelax": _abi.MJ_MC_OVERRELAX}


@dataclass
class MCInput:
    """IO-input/MC_io.f90:8-35 (one sampling method, as rw_MC requires)."""
    n_Tsteps: int = 1
    n_sizerelax: int = 1
    N_relaxation: int = 1000
    T_relax: int = 1
    T_auto: int = 1
    Total_MC_Steps: int = 1000
    cone: float = math.pi
    sampling: str = "sphere"

    def __post_init__(self):
        if self.sampling not in SAMPLING:
            raise ValueError(f"sampling must be one of {sorted(SAMPLING)}")


def temperatures(T_ini: float, T_fin: float, n: int, geometric: bool = False) -> np.ndarray:
    """ini_temp (Metropolis-MC/initialize_temperature.f90:14-50), in Kelvin."""
    if n <= 1:
        return np.array([T_ini], np.float64)
    i = np.arange(n, dtype=np.float64)
    if geometric:
        return (T_fin / T_ini) ** (i / (n - 1)) * T_ini
    return (T_fin - T_ini) / (n - 1) * i + T_ini


class MetropolisMC:
    """The Monte Carlo chain of one spin configuration on the device."""

    def __init__(self, ham: Hamiltonian, sampling: str = "sphere", cone: float = math.pi, seed: int = 0,
                 stream_id: int = 0, adapt_cone: bool = True, track_totals: bool = False):
        """track_totals: the recorded energies and summed spins are the totals of
        the call's start updated by every accepted move (track_val's E_total and
        Magnetization, MCstep.f90:60-68) instead of recomputed after every sweep."""
        if sampling not in SAMPLING:
            raise ValueError(f"sampling must be one of {sorted(SAMPLING)}")
        self.ham = ham
        self.p = _abi.McParams(0.0, float(cone), SAMPLING[sampling], int(bool(adapt_cone)), int(seed),
                               int(stream_id), 0, 0, 0, 0, int(bool(track_totals)))
        self.colors = (0, 0, 0, 0)  # {q, b, c, 1} linear or {cx, cy, cz, 0} product, set by sweeps

    @property
    def cone(self) -> float:
        return self.p.cone

    @property
    def rate(self) -> float:
        """accepted / proposed moves so far (track_val%rate)."""
        return self.p.accepted_total / self.p.proposed_total if self.p.proposed_total else 0.0

    def sweeps(self, m, nsweeps: int, temperature: float, record: bool = True):
        """nsweeps sweeps at `temperature` (K) on m, a CUDA (3, N) tensor updated in
        place.  Returns (E (nsweeps,), summed spins (nsweeps, 3), accepted) with E and
        the sums after each sweep as CUDA tensors (None when record is False)."""
        import torch

        assert _is_torch(m) and m.is_contiguous() and m.shape == (3, self.ham.N) and m.dtype == torch.float64
        self.p.temperature = float(temperature)
        E = torch.empty(nsweeps, dtype=torch.float64, device=m.device) if record else None
        Mg = torch.empty((nsweeps, 3), dtype=torch.float64, device=m.device) if record else None
        acc = C.c_int64()
        col = np.zeros(4, np.int32)
        check(lib.mj_mc_sweeps(self.ham.plan, ptr(m), C.byref(self.p), int(nsweeps), ptr(E), ptr(Mg), C.byref(acc),
                               col.ctypes.data_as(C.POINTER(C.c_int32)), _stream(m)))
        self.colors = tuple(int(c) for c in col)
        return E, Mg, acc.value


@dataclass
class ThermVal:
    """therm_val (Metropolis-MC/thermo_val.f90:16-33), the columns this library fills."""
    T: float
    E: float
    E_err: float
    C: float
    M: np.ndarray
    M_err: np.ndarray
    chi_M: np.ndarray


def therm_set(T: float, E_samples: Sequence[float], M_samples, nsites: int) -> ThermVal:
    """Averages of Total_MC_Steps measurements of the total energy and summed
    spins at T (K) (thermo_val.f90:44-77: C and chi per site in units of 1/kT,
    the *_err columns the per-site sample standard deviation)."""
    E = np.asarray(E_samples, np.float64)
    M = np.asarray(M_samples, np.float64).reshape(-1, 3)
    n = E.shape[0]
    kT = T * KB
    av_site, av_n, av_kt = 1.0 / nsites, 1.0 / n, 1.0 / kT
    E_sum, E_sq = E.sum(), (E * E).sum()
    M_sum, M_sq = M.sum(0), (M * M).sum(0)
    C_ = (E_sq * av_n - (E_sum * av_n) ** 2) * av_kt ** 2 * av_site
    chi = (M_sq * av_n - (M_sum * av_n) ** 2) * av_kt * av_site
    E_err, M_err = 0.0, np.zeros(3)
    if n > 1:
        E_err = math.sqrt(abs(E_sq - E_sum ** 2 * av_n) / (n - 1)) * av_site
        M_err = np.sqrt(np.abs(M_sq - M_sum ** 2 * av_n) / (n - 1)) * av_site
    return ThermVal(T, E_sum * av_n * av_site, E_err, C_, M_sum * av_n * av_site, M_err, chi)


EM_HEADER_COLUMNS = ['# 1:T', '2:E_av', '3:E_err', '4:C', '5:M', '6:Mx', '7:My', '8:Mz', '9:M_err_x', '10:M_err_y',
                     '11:M_err_z', '12:chi_x', '13:chi_y', '14:chi_z', '15:vx', '16:vy', '17:vz', '18:qeuler',
                     '19:Chi_q', '20:Q+', '21:Chi_qp', '22:Q-', '23:Chi_qm', '24:l_x', '25:l_y', '26:l_z',
                     '27:Chi_QpQm', '28: Re(Mj+Mi-)', '29: Im(Mj+Mi-)', '30: Re(Mi+Mi+)', '31: Im(Mi+Mi+)',
                     '32: Re(Mi+Mi-)', '33: Re(Mi+Mj+)', '34: Im(Mi+Mj+)']


def thermo_print(path: str, rows: List[ThermVal]) -> None:
    """EM.dat of the Monte Carlo (thermo_val.f90:88-129): the header of
    thermo_print_init, then per temperature 35 values in (E20.10E3, 2X)."""
    from .reference_io import fortran_e

    with open(path, "w") as f:
        f.write("".join(c + " " * 15 for c in EM_HEADER_COLUMNS) + "\n")
        for r in rows:
            vals = [r.T, r.E, r.E_err, r.C, float(np.linalg.norm(r.M)), *r.M, *r.M_err, *r.chi_M]
            vals += [0.0] * (35 - len(vals))
            f.write("".join(fortran_e(v, 20, 10, 3) + "  " for v in vals[:34]) + fortran_e(vals[34], 20, 10, 3) + "\n")


def montecarlo_run(ham: Hamiltonian, m, inp: MCInput, temps: Sequence[float], seed: int = 0,
                   chain: Optional[MetropolisMC] = None) -> List[ThermVal]:
    """The temperature loop of Metropolis-MC/MonteCarlo.f90:128-160 on m (CUDA
    (3, N), in place): per temperature N_relaxation * T_relax relaxation sweeps,
    then Total_MC_Steps measurements of (E, summed spins), each after T_auto
    sweeps, the totals tracked through the accepted moves as track_val does.
    The chain (cone, counts) carries over from one temperature to the next."""
    chain = chain or MetropolisMC(ham, inp.sampling, inp.cone, seed, track_totals=True)
    out = []
    for T in temps:
        chain.sweeps(m, max(1, inp.N_relaxation * max(1, inp.T_relax)), T, record=False)
        n = inp.Total_MC_Steps * max(1, inp.T_auto)
        E, Mg, _ = chain.sweeps(m, n, T, record=True)
        every = max(1, inp.T_auto)
        E = E[every - 1::every].cpu().numpy()
        Mg = Mg[every - 1::every].cpu().numpy()
        out.append(therm_set(T, E, Mg, ham.N))
    return out


def parallel_tempering_run(batch, inp: MCInput, seed: int = 0, stream_id: int = 0, adapt_cone: bool = True,
                           return_series: bool = False):
    """The swap loop of paratemp-MC/parallel_tempering.f90:163-181 on a
    ReplicaBatch whose replicas (all of one size) hold the temperature ladder:
    n_sizerelax rounds of T_auto sweeps of every replica, each round measured
    (measure_add, the measurement following the temperature) and followed by a
    swap round.  Returns the ThermVal of every ladder temperature, ascending
    (and, with return_series, the per-round energies, summed spins and ladder
    slots of every replica).  The reference's temperature-set optimisation (N_Topt > 1,
    calculate_diffusion) is not run: one pass over the ladder, as N_Topt = 1."""
    p = _abi.McParams(0.0, float(inp.cone), SAMPLING[inp.sampling], int(bool(adapt_cone)), int(seed), int(stream_id),
                      0, 0, 0, 0, 0)
    n = max(1, inp.n_sizerelax)
    E, M, S = batch.monte_carlo(p, n, max(1, inp.T_auto), swap=True)
    E, M, S = E.cpu().numpy(), M.cpu().numpy(), S.cpu().numpy()
    T_rep, _ = batch.temperatures()
    ladder = np.sort(T_rep)
    nsite = int(batch.sizes[0, 0] * batch.sizes[0, 1])
    out = []
    for l, T in enumerate(ladder):
        sel = S == l
        out.append(therm_set(float(T), E[sel], M[sel], nsite))
    return (out, (E, M, S)) if return_series else out
