"""The reference's file formats: the `input` deck, order-parameter files and
the dynamics outputs, so that a run of this library can be set up from a
Matjes input directory and diffed against a reference run.

Input deck (a subset of the keywords Matjes reads, same meaning):
  lattice        Periodic_log, alat, lattice (3 rows), rotate_lattice, Nsize
                 (IO-input/rw_lattice.f90:28-80: each lattice row is normalised
                 and its length folded into alat; the rotation is Z-X-Z Euler in
                 units of pi)
  cell           atomtypes N + N lines `name moment charge mass use_ph [orbitals]`
                 (IO-utils/io-utils.f90:895-944), atoms N + N lines
                 `name|type-id x y z [div]` in lattice coordinates
                 (io-utils.f90:828-890)
  Hamiltonian    magnetic_J block `t1 t2 shell J` (get_H_pair, io-utils.f90:584-660:
                 lines until one does not parse, '#' lines skipped, zero values
                 dropped, types ordered t1 <= t2), magnetic_D block
                 `t1 t2 mediator shell D` (get_H_triple), magnetic_anisotropy block
                 `type ex ey ez K` or `type kx ky kz` (Energy/anisotropy_heisenberg.f90:
                 12-56: the 3-real form takes |k| as magnitude with the sign of the
                 last non-zero component), H_ext, enable_H, c_H_J, c_H_D, c_H_ani,
                 c_zeeman, mag_dip_use, mag_dip_period_cut
  dynamics       integration, timestep, duration, damping, Efreq, Tini, Tfin
                 (IO-input/dyna_io.f90:56-59, rw_extpar.f90:34-38,
                 solvers/solver_commun.f90:57)
  minimisation   steps, masse, timestep, min_Efreq, convergence_criteria
                 (IO-input/minimize_io.f90:40-44)
  Monte Carlo    simulation (metropolis | parallel-tempering), n_Tsteps, Tini, Tfin,
                 n_relaxation, T_relax, T_auto, Total_MC_Steps, n_sizerelax, cone and
                 one of the logicals ising, underrelaxation, overrelaxation,
                 sphere_samp, equi_samp (IO-input/MC_io.f90:92-150); run_montecarlo
                 writes the Monte Carlo EM.dat (thermo_val.f90 thermo_print)
Values follow Fortran list-directed input: `1.0d-3` exponents, logicals
`.T.`/`T`/`.true.`, trailing text after the values ignored.

Files:
  <name>_init.dat  3N values in site order, any layout (order_parameter.f90:140-175:
                   fewer or more values than the lattice holds is an error)
  <name>_<tag>.dat one site per line, 3 x E24.16 then two blanks (write_config.f90:
                   62-81, io-utils.f90:227-237)
  Beff_<tag>.dat   one site per line, 3 x (E20.12E3, 2 blanks) (print_Beff.f90:10-29)
  EM.dat           header line of 19 names, then per Efreq step
                   I12, 18 x E20.12E3 (dynamics/spindynamics.f90:135-139, 336-360):
                   step, time, E per cell, |M|, M, |vorticity|, vorticity, q, q+,
                   q-, T, measured T, H; the topological columns carry the
                   reference's placeholder values (it computes them only with
                   calc_topo)
"""
from __future__ import annotations

import math
import os
import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .deck import Deck

# ----------------------------------------------------------------------
# Fortran list-directed values


def fortran_float(tok: str) -> float:
    return float(tok.replace("d", "e").replace("D", "E"))


def fortran_bool(tok: str) -> bool:
    t = tok.strip().lstrip(".").upper()
    if t.startswith("T"):
        return True
    if t.startswith("F"):
        return False
    raise ValueError(f"not a Fortran logical: {tok!r}")


def _tokens(line: str) -> List[str]:
    return [t for t in re.split(r"[\s,]+", line.strip()) if t]


def fortran_e(x: float, w: int, d: int, e: Optional[int] = None) -> str:
    """Fortran Ew.d[Ee] output of x (mantissa 0.d...d, exponent of e digits,
    2 when e is not given), right-justified in w characters."""
    if not math.isfinite(x):
        return ("NaN" if math.isnan(x) else ("-Infinity" if x < 0 else "Infinity")).rjust(w)
    neg = math.copysign(1.0, x) < 0  # gfortran writes the sign of a negative zero
    a = abs(x)
    if a == 0.0:
        digits, ex = "0" * d, 0
    else:
        s = f"{a:.{d - 1}e}"
        mant, ep = s.split("e")
        digits = mant.replace(".", "")
        ex = int(ep) + 1
    ed = e if e is not None else 2
    if e is None and abs(ex) > 99:
        exp = f"{'+' if ex >= 0 else '-'}{abs(ex):03d}"
    else:
        exp = f"E{'+' if ex >= 0 else '-'}{abs(ex):0{ed}d}"
    return (("-" if neg else "") + "0." + digits + exp).rjust(w)


# ----------------------------------------------------------------------
# the input deck


class InputDeck:
    """The lines of a Matjes `input` file, searched the way set_pos_entry does:
    the first non-comment line whose first token is the keyword."""

    def __init__(self, text: str):
        self.lines = text.splitlines()

    @classmethod
    def read(cls, path: str) -> "InputDeck":
        with open(path) as f:
            return cls(f.read())

    def find(self, key: str) -> Optional[int]:
        for i, ln in enumerate(self.lines):
            s = ln.strip()
            if not s or s.startswith("#"):
                continue
            t = _tokens(s)
            if t and t[0] == key:
                return i
        return None

    def values(self, key: str, n: int, conv=fortran_float, default=None):
        i = self.find(key)
        if i is None:
            return default
        t = _tokens(self.lines[i])[1:]
        if len(t) < n:
            raise ValueError(f"keyword {key}: expected {n} values")
        vals = [conv(x) for x in t[:n]]
        return vals if n > 1 else vals[0]

    def rows(self, key: str, n: int, conv=fortran_float):
        """n lines after the keyword line (matrix inputs like `lattice`)."""
        i = self.find(key)
        if i is None:
            return None
        out = []
        for ln in self.lines[i + 1:i + 1 + n]:
            out.append([conv(x) for x in _tokens(ln)[:3]])
        return out

    def block(self, key: str, nint: int, nreal: int):
        """Lines after the keyword with nint integers then nreal reals, until a
        line that does not parse; '#' lines are skipped."""
        i = self.find(key)
        if i is None:
            return None
        out = []
        for ln in self.lines[i + 1:]:
            s = ln.strip()
            if s.startswith("#"):
                continue
            t = _tokens(s)
            try:
                ints = [int(x) for x in t[:nint]]
                reals = [fortran_float(x) for x in t[nint:nint + nreal]]
            except (ValueError, IndexError):
                break
            if len(ints) < nint or len(reals) < nreal:
                break
            out.append((ints, reals))
        return out

    def counted(self, key: str) -> Optional[Tuple[int, List[str]]]:
        """`key N` followed by N lines (atomtypes, atoms)."""
        i = self.find(key)
        if i is None:
            return None
        t = _tokens(self.lines[i])
        n = int(t[1])
        return n, self.lines[i + 1:i + 1 + n]


@dataclass
class DynamicsInput:
    integration: int = 1
    timestep: float = 0.1
    duration: int = 1
    damping: float = 0.0
    Efreq: int = 1
    Tini: float = 0.0
    Tfin: float = 0.0


@dataclass
class MinimizeInput:
    mass: float = 1.0
    timestep: float = 0.1
    steps: int = 2 ** 62
    Efreq: int = 100
    conv_torque: float = 1e-6


@dataclass
class ReferenceInput:
    deck: Deck
    dynamics: DynamicsInput
    minimize: MinimizeInput
    atom_names: List[str] = field(default_factory=list)
    simulation: str = ""
    # the Monte Carlo input (IO-input/MC_io.f90 rw_MC), None when the deck sets
    # no sampling method
    monte_carlo: Optional[object] = None
    # the GNEB input (IO-input/GNEB_io.f90 rw_gneb)
    gneb: Optional[object] = None


MC_SAMPLING_KEYS = (("ising", "ising"), ("underrelaxation", "underrelax"), ("overrelaxation", "overrelax"),
                    ("sphere_samp", "sphere"), ("equi_samp", "equi"))


def parse_monte_carlo(inp: "InputDeck"):
    """rw_MC (IO-input/MC_io.f90:92-150): the counts and the sampling method.
    A logical keyword needs its value (`ising .T.`), as get_bool reads it; more
    than one method is an error, none gives None."""
    from .montecarlo import MCInput

    methods = [name for key, name in MC_SAMPLING_KEYS if inp.values(key, 1, fortran_bool, False)]
    if len(methods) > 1:
        raise ValueError(f"more than one Monte Carlo sampling method set: {methods}")
    if not methods:
        return None
    return MCInput(n_Tsteps=inp.values("n_Tsteps", 1, int, 1), n_sizerelax=inp.values("n_sizerelax", 1, int, 1),
                   N_relaxation=inp.values("n_relaxation", 1, int, 1000), T_relax=inp.values("T_relax", 1, int, 1),
                   T_auto=inp.values("T_auto", 1, int, 1), Total_MC_Steps=inp.values("Total_MC_Steps", 1, int, 1000),
                   cone=inp.values("cone", 1, default=math.pi), sampling=methods[0])


def parse_gneb(inp: "InputDeck"):
    """rw_gneb (IO-input/GNEB_io.f90:43-112): the GNEB keywords with their
    defaults; initpath sets read_path / read_outer / min_type (-1: unchanged;
    1: geodesic path, no minimisation; 2: path read, minimize; 3: path read,
    minimize_infdamp; other values: geodesic path, minimize_infdamp), the
    gnebinit_* keywords override them."""
    from .gneb import GNEBInput

    d = GNEBInput()
    g = GNEBInput(
        momfile_i=inp.values("momfile_i", 1, str, d.momfile_i), momfile_f=inp.values("momfile_f", 1, str, d.momfile_f),
        restartfile_path=inp.values("restartfile_path", 1, str, d.restartfile_path),
        spring=inp.values("spring", 1, default=d.spring), initpath=inp.values("initpath", 1, int, d.initpath),
        amp_rnd=inp.values("amp_rnd", 1, default=d.amp_rnd),
        amp_rnd_path=inp.values("amp_rnd_path", 1, default=d.amp_rnd_path),
        itrmax=inp.values("mep_itrmax", 1, int, d.itrmax), every=inp.values("meptraj_step", 1, int, d.every),
        mepftol=inp.values("mep_ftol", 1, default=d.mepftol),
        mepftol_ci=inp.values("mep_ftol_ci", 1, default=d.mepftol_ci),
        do_gneb=bool(inp.values("do_gneb_simple", 1, fortran_bool, d.do_gneb)),
        do_gneb_ci=bool(inp.values("do_gneb_ci", 1, fortran_bool, d.do_gneb_ci)),
        do_norm_rx=inp.values("do_norm_rx", 1, str, d.do_norm_rx), en_zero=inp.values("en_zero", 1, str, d.en_zero),
        dt=inp.values("vpo_dt", 1, default=d.dt), mass=inp.values("vpo_mass", 1, default=d.mass),
        sample_num=inp.values("sample_num", 1, int, d.sample_num), nim=inp.values("nim", 1, int, d.nim))
    if g.initpath == 1:
        g.read_path, g.read_outer, g.min_type = False, True, 0
    elif g.initpath == 2:
        g.read_path, g.read_outer, g.min_type = True, True, 2
    elif g.initpath == 3:
        g.read_path, g.read_outer, g.min_type = True, True, 1
    elif g.initpath != -1:
        g.read_path, g.read_outer, g.min_type = False, True, 1
    g.read_path = bool(inp.values("gnebinit_read_path", 1, fortran_bool, g.read_path))
    g.read_outer = bool(inp.values("gnebinit_read_outer", 1, fortran_bool, g.read_outer))
    g.min_type = inp.values("gnebinit_min_type", 1, int, g.min_type)
    return g


def _rotation_zxz(angles_pi: Sequence[float]) -> np.ndarray:
    """Z-X-Z Euler rotation, angles in units of pi (rw_lattice.f90:40-60)."""
    a1, a2, a3 = (np.pi * float(x) for x in angles_pi)
    s1, s2, s3, c1, c2, c3 = np.sin(a1), np.sin(a2), np.sin(a3), np.cos(a1), np.cos(a2), np.cos(a3)
    return np.array([[c1 * c3 - c2 * s1 * s3, -c1 * s3 - c2 * c3 * s1, s1 * s2],
                     [c3 * s1 + c1 * c2 * s3, c1 * c2 * c3 - s1 * s3, -c1 * s2],
                     [s2 * s3, c3 * s2, c2]])


def parse_input(path_or_text: str) -> ReferenceInput:
    """A Matjes `input` deck (file path or its text) as a Deck plus the dynamics
    and minimisation parameters."""
    text = open(path_or_text).read() if os.path.exists(path_or_text) else path_or_text
    inp = InputDeck(text)
    periodic = inp.values("Periodic_log", 3, fortran_bool, [True, True, True])
    alat = np.array(inp.values("alat", 3, default=[1.0, 1.0, 1.0]), float)
    net = inp.rows("lattice", 3)
    net = np.eye(3) if net is None else np.array(net, float)
    for j in range(3):
        ss = np.linalg.norm(net[j])
        if ss < 1e-8:
            raise ValueError("lattice vectors are degenerate")
        net[j] /= ss
        alat[j] *= ss
    rot = inp.values("rotate_lattice", 3, default=None)
    if rot is not None and any(r != 0.0 for r in rot):
        net = net @ _rotation_zxz(rot)
    areal = net * alat[:, None]
    L = inp.values("Nsize", 3, int, [1, 1, 1])

    types = inp.counted("atomtypes")
    names, moments = [], []
    if types is not None:
        for ln in types[1]:
            t = _tokens(ln)
            names.append(t[0])
            moments.append(fortran_float(t[1]))
    atoms = []
    cell = inp.counted("atoms")
    if cell is not None:
        for ln in cell[1]:
            t = _tokens(ln)
            pos = [fortran_float(x) for x in t[1:4]]
            if len(t) >= 5:
                try:
                    div = int(t[4])
                    pos = [p / div for p in pos]
                except ValueError:
                    pass
            try:
                tid = int(t[0])
            except ValueError:
                if t[0] not in names:
                    raise ValueError(f"atom {t[0]} is not among the atom types")
                tid = names.index(t[0]) + 1
            atoms.append((tuple(pos), tid, moments[tid - 1] if moments else 0.0))

    J = []
    for ints, reals in inp.block("magnetic_J", 3, 1) or []:
        t1, t2, shell = ints
        if reals[0] == 0.0:
            continue
        J.append((min(t1, t2), max(t1, t2), shell, reals[0]))
    D = []
    for ints, reals in inp.block("magnetic_D", 4, 1) or []:
        t1, t2, tm, shell = ints
        if reals[0] == 0.0:
            continue
        D.append((t1, t2, tm, shell, reals[0]))
    K = []
    blk4 = inp.block("magnetic_anisotropy", 1, 4)
    if blk4:
        for ints, reals in blk4:
            if any(r != 0.0 for r in reals):
                K.append((ints[0], tuple(reals[:3]), reals[3]))
    else:
        for ints, reals in inp.block("magnetic_anisotropy", 1, 3) or []:
            if all(r == 0.0 for r in reals):
                continue
            mag = float(np.linalg.norm(reals))
            for r in reals:  # the sign of the last non-zero component
                if r != 0.0:
                    mag = math.copysign(mag, r)
            K.append((ints[0], tuple(reals), mag))

    deck = Deck(L=tuple(L), periodic=tuple(int(p) for p in periodic), areal=areal, atoms=atoms, J=J, D=D, K=K,
                B_ext=tuple(inp.values("H_ext", 3, default=[0.0, 0.0, 0.0])),
                zeeman_on=bool(inp.values("enable_H", 1, fortran_bool, False)),
                dip=bool(inp.values("mag_dip_use", 1, fortran_bool, False)),
                dip_cut=tuple(inp.values("mag_dip_period_cut", 3, int, [1, 1, 1])),
                c_H_J=inp.values("c_H_J", 1, default=-1.0), c_H_D=inp.values("c_H_D", 1, default=-1.0),
                c_H_ani=inp.values("c_H_ani", 1, default=1.0), c_zeeman=inp.values("c_zeeman", 1, default=-1.0))
    dyn = DynamicsInput(integration=inp.values("integration", 1, int, 1),
                        timestep=inp.values("timestep", 1, default=0.1),
                        duration=inp.values("duration", 1, int, 1), damping=inp.values("damping", 1, default=0.0),
                        Efreq=inp.values("Efreq", 1, int, 1), Tini=inp.values("Tini", 1, default=0.0),
                        Tfin=inp.values("Tfin", 1, default=0.0))
    mn = MinimizeInput(mass=inp.values("masse", 1, default=1.0), timestep=inp.values("timestep", 1, default=0.1),
                       steps=inp.values("steps", 1, int, 2 ** 62), Efreq=inp.values("min_Efreq", 1, int, 100),
                       conv_torque=inp.values("convergence_criteria", 1, default=1e-6))
    sim = inp.values("simulation", 1, str, "")
    return ReferenceInput(deck=deck, dynamics=dyn, minimize=mn, atom_names=names, simulation=sim,
                          monte_carlo=parse_monte_carlo(inp), gneb=parse_gneb(inp))


# ----------------------------------------------------------------------
# order-parameter files


def read_order_file(path: str, nsites: int, dim: int = 3) -> np.ndarray:
    """<name>_init.dat: exactly dim * nsites values in site order, any layout."""
    vals = []
    with open(path) as f:
        for ln in f:
            vals.extend(fortran_float(t) for t in _tokens(ln))
    if len(vals) < dim * nsites:
        raise ValueError(f"{path}: unexpected end of file (lattice of {nsites} sites)")
    if len(vals) > dim * nsites:
        raise ValueError(f"{path}: unexpected further entries (lattice of {nsites} sites)")
    return np.array(vals, float).reshape(nsites, dim)


def write_order_file(path: str, m: np.ndarray) -> None:
    """<name>_<tag>.dat: one site per line, dim x E24.16 then two blanks."""
    m = np.asarray(m, float).reshape(len(m), -1)
    with open(path, "w") as f:
        for row in m:
            f.write("".join(fortran_e(float(v), 24, 16) for v in row) + "  \n")


def write_beff(path: str, B: np.ndarray) -> None:
    """Beff_<tag>.dat: one site per line, dim x (E20.12E3, 2 blanks)."""
    B = np.asarray(B, float).reshape(len(B), -1)
    with open(path, "w") as f:
        for row in B:
            f.write("".join(fortran_e(float(v), 20, 12, 3) + "  " for v in row) + "\n")


EM_HEADER = ['# 1:step', '2:real_time (fs)', '3:E_av (eV)', '4:M', '5:Mx', '6:My', '7:Mz', '8:vorticity', '9:vx',
             '10:vy', '11:vz', '12:qeuler', '13:q+', '14:q-', '15:T= (K)', '16:Tfin=', '17:Hx (T)', '18:H (T)y=',
             '19:H (T)z=']
# the values the reference writes in the topology columns without calc_topo:
# dumy = 1.2345789d+98*pi*4.0d0, q = dumy/pi/4.0d0; dumy(3:5) = 1.2345789d+98*3.0*sqrt(3.0)
# (single-precision 3.0 and sqrt), vorticity = dumy/3.0d0/sqrt(3.0d0)
_Q_UNSET = 1.2345789e98 * math.pi * 4.0 / math.pi / 4.0
_V_UNSET = 1.2345789e98 * 3.0 * float(np.sqrt(np.float32(3.0))) / 3.0 / math.sqrt(3.0)


def em_header() -> str:
    return "".join(f"{h}  " for h in EM_HEADER) + "\n"


def em_line(step: int, time_fs: float, E_per_cell: float, M: Sequence[float], T: float, T_measured: float,
            H: Sequence[float], topo: Optional[Tuple[float, float, Sequence[float]]] = None) -> str:
    """One EM.dat row; topo = (q+, q-, vorticity vector) when computed."""
    if topo is None:
        qp = qm = _Q_UNSET
        vort = [_V_UNSET] * 3
    else:
        qp, qm, vort = topo
    Mn = float(np.linalg.norm(M))
    vals = [time_fs, E_per_cell, Mn, *M, float(np.linalg.norm(vort)), *vort, qp + qm, qp, qm, T, T_measured, *H]
    return f"{step:12d}" + "".join(fortran_e(float(v), 20, 12, 3) + "  " for v in vals[:-1]) + \
        fortran_e(float(vals[-1]), 20, 12, 3) + "\n"


# ----------------------------------------------------------------------
# a dynamics run set up from an input directory


def run_dynamics(directory: str, integrator: Optional[str] = None, seed: int = 1, write: bool = True):
    """spindynamics_run of an input directory on the GPU: reads `input`,
    `magnetic_init.dat` and `Bfield_init.dat` when present, runs `duration`
    steps, writes EM.dat every Efreq steps and magnetic_final.dat
    (dynamics/spindynamics.f90:135-139, 260-360).  integration 1 = Euler,
    2 = Heun (Matjes), 3 = SIB."""
    import torch

    from . import Hamiltonian, SpinDynamics
    from .deck import random_sphere
    from ._abi import C, check, lib

    ri = parse_input(os.path.join(directory, "input"))
    deck, dyn = ri.deck, ri.dynamics
    ham = Hamiltonian(deck)
    N = deck.nsites
    init = os.path.join(directory, "magnetic_init.dat")
    m0 = read_order_file(init, N) if os.path.exists(init) else random_sphere(N, seed)
    bf = os.path.join(directory, "Bfield_init.dat")
    if os.path.exists(bf):
        ham.set_bfield(read_order_file(bf, deck.ncell))
    name = integrator or {1: "euler", 2: "heun", 3: "sib"}.get(dyn.integration, "euler")
    sd = SpinDynamics(ham, integrator=name, timestep=dyn.timestep, alpha=dyn.damping, temperature=dyn.Tini,
                      noise="philox" if dyn.Tini > 0 else "off", seed=seed)
    m = torch.tensor(m0.T.copy(), device="cuda")
    lines = [em_header()]
    Ef = max(1, dyn.Efreq)
    for j in range(1, dyn.duration + 1):
        sd.run(m, 1, step0=j - 1)
        if (j - 1) % Ef == 0:
            mh = m.cpu().numpy().T
            E = ham.energy(mh) / deck.ncell
            Tm = C.c_double()
            st = None
            if dyn.Tini * dyn.damping > 0:
                from .hamiltonian import SpinState

                st = SpinState(ham, mh)
                check(lib.mj_measure_temperature(ham.plan, st.handle, C.byref(Tm)))
            lines.append(em_line(j, j * dyn.timestep, E, mh.sum(0) / deck.ncell, dyn.Tini, Tm.value,
                                 deck.B_ext))
    mT = m.cpu().numpy().T.copy()
    if write:
        with open(os.path.join(directory, "EM.dat"), "w") as f:
            f.writelines(lines)
        write_order_file(os.path.join(directory, "magnetic_final.dat"), mT)
    return mT, lines


def run_montecarlo(directory: str, seed: int = 1, write: bool = True):
    """The Monte Carlo of an input directory on the GPU: reads `input` and
    `magnetic_init.dat` when present (else a random state from `seed`), the
    temperatures of ini_temp (Tini .. Tfin in n_Tsteps steps, geometric when a
    file `geometric` is in the directory, Metropolis-MC/initialize_temperature.f90),
    then `simulation metropolis` runs montecarlo_run (Metropolis-MC/MonteCarlo.f90)
    on one lattice, `simulation parallel-tempering` runs parallel_tempering_run
    (paratemp-MC/parallel_tempering.f90) on n_Tsteps replicas of the lattice.
    Writes EM.dat (thermo_print) and returns the ThermVal rows."""
    import torch

    from . import Hamiltonian
    from .batch import ReplicaBatch
    from .deck import random_sphere
    from .montecarlo import montecarlo_run, parallel_tempering_run, temperatures, thermo_print

    ri = parse_input(os.path.join(directory, "input"))
    inp = ri.monte_carlo
    if inp is None:
        raise ValueError("the input sets no Monte Carlo sampling method (ising, underrelaxation, overrelaxation, "
                         "sphere_samp or equi_samp)")
    deck = ri.deck
    N = deck.nsites
    init = os.path.join(directory, "magnetic_init.dat")
    m0 = read_order_file(init, N) if os.path.exists(init) else random_sphere(N, seed)
    temps = temperatures(ri.dynamics.Tini, ri.dynamics.Tfin, inp.n_Tsteps,
                         geometric=os.path.exists(os.path.join(directory, "geometric")))
    if ri.simulation == "parallel-tempering":
        n = len(temps)
        batch = ReplicaBatch(deck, [deck.L[:2]] * n, np.tile(np.asarray(deck.B_ext, float), (n, 1)), temps)
        batch.upload(np.tile(m0, (n, 1)))
        rows = parallel_tempering_run(batch, inp, seed=seed)
    elif ri.simulation == "metropolis":
        ham = Hamiltonian(deck)
        m = torch.tensor(m0.T.copy(), device="cuda")
        rows = montecarlo_run(ham, m, inp, temps, seed=seed)
    else:
        raise ValueError(f"simulation {ri.simulation!r} is not a Monte Carlo (metropolis, parallel-tempering)")
    if write:
        thermo_print(os.path.join(directory, "EM.dat"), rows)
    return rows


def run_gneb(directory: str, seed: int = 0, write: bool = True) -> dict:
    """The GNEB of an input directory on the GPU (`simulation GNEB`, GNEB_run of
    GNEB/gneb.f90): reads `input` (the lattice, Hamiltonian, GNEB and
    minimisation keywords), the initial and final states momfile_i / momfile_f
    (read_outer) and the path <restartfile_path>_<k>.dat, k = 1 .. nim
    (read_path), each as an order-parameter file of the lattice; then
    gneb.gneb_run, writing en_path.in, en_path.out, enfit_path.out,
    ensp_path.out, image-GNEB_<k>.dat, image-GNEB-saddlepoint.dat and
    SpinSTM_GNEB_ini.dat / SpinSTM_GNEB_fin.dat into the directory."""
    from .gneb import gneb_run

    ri = parse_input(os.path.join(directory, "input"))
    if ri.simulation != "GNEB":
        raise ValueError(f"simulation {ri.simulation!r} is not GNEB")
    g = ri.gneb
    deck = ri.deck
    N = deck.nsites

    def read(name):
        return read_order_file(os.path.join(directory, name), N)

    m_i = read(g.momfile_i) if g.read_outer else None
    m_f = read(g.momfile_f) if g.read_outer else None
    path = np.stack([read(f"{g.restartfile_path}_{k}.dat") for k in range(1, g.nim + 1)]) if g.read_path else None
    return gneb_run(deck, g, m_i, m_f, path, minimize_input=ri.minimize, directory=directory if write else None,
                    seed=seed)
