"""Extract the reference's minimisation test into a fixture.

    python tests/golden/make_golden_minimization.py <Matjes source tree>

Reads tests/serial/minimization/ of the Matjes source tree and writes
minimization_triangular100.json and minimization_triangular100.npz beside this
script.  The run is a 100 x 100 triangular monolayer (one magnetic atom per cell,
a non-magnetic atom at the hollow site (2/3, 1/3, -0.76) that mediates the DMI)
with ten exchange shells, nearest-neighbour DMI, an easy axis and a 20 T field;
its log (REF) gives the energy of the start state (SpinSTMi.dat) and of each of
the 406 iterates of the minimiser down to a torque of 1e-5.

The deck is in the legacy keyword format that predates the current `input`
parser; each keyword is mapped here onto the current one (the values are
unchanged):

  Nsize 100 100 1            -> Nsize (L = 100 x 100 x 1)
  lattice (3 rows), alat 1   -> lattice vectors a1 = (1/2, -sqrt3/2, 0),
                                a2 = (1/2, sqrt3/2, 0), a3 = (0, 0, 1), in nm
  motif row 1: 0 0 0 3.0     -> magnetic atom, type 1, moment mu_s = 3 mu_B
  motif row 2: 2/3 1/3 -0.76 0.0 -> non-magnetic atom, type 2 (DMI mediator)
  Periodic_log .T. .T. .T.   -> periodic in-plane; the single layer gets no
                                neighbours along z (the log's start energy
                                -0.067544 eV/cell holds only without them:
                                with the images of the layer along z it is
                                -0.0961)
  J_k v (k = 1..10)          -> magnetic_J 1 1 k v (eV, c_H_J = -1)
  DM v 0 0                   -> magnetic_D 1 1 2 1 v (shell 1, mediator type 2)
  EA 0 0 1, D_ani v 0 0      -> magnetic_anisotropy 1 0 0 1 v (c_H_ani = +1,
                                v < 0: easy axis)
  H_ext 0 0 20               -> H_ext 0 0 20 (T, Zeeman on)

SpinSTMi.dat holds x y z mx my mz per cell (8 decimals), a2 fastest; the
spins are stored here as integers k = round(1e8 m) in the site order of the
current code (x fastest along a1): k / 1e8 is the double the reference parses.
"""
import json
import os
import re
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit(__doc__)
base = os.path.join(sys.argv[1], "tests", "serial", "minimization")
HERE = os.path.dirname(os.path.abspath(__file__))


def keywords(path):
    out = {}
    for line in open(path):
        line = line.split("#")[0].strip()
        if line:
            w = line.split()
            out[w[0]] = w[1:]
    return out


def fnum(s):
    return float(s.lower().replace("d", "e"))


inp = keywords(os.path.join(base, "inp"))
lat_lines = [l.split() for l in open(os.path.join(base, "lattice.in")) if l.strip() and not l.startswith("#")]
L = [int(x) for x in lat_lines[0][1:4]]
rows = {i: [float(x) for x in lat_lines[i]] for i in range(len(lat_lines)) if re.match(r"^-?[0-9.]+$", lat_lines[i][0])}
vec = [rows[i] for i in sorted(rows)[:3]]
motif = [rows[i] for i in sorted(rows)[3:5]]
Js = [fnum(inp[f"J_{k}"][0]) for k in range(1, 11)]
deck = {
    "L": L, "periodic": [1, 1, 0], "areal": vec,
    "atoms": [[motif[0][:3], 1, motif[0][3]], [motif[1][:3], 2, motif[1][3]]],
    "J": [[1, 1, k + 1, v] for k, v in enumerate(Js)],
    "D": [[1, 1, 2, 1, fnum(inp["DM"][0])]],
    "K": [[1, [fnum(x) for x in inp["EA"]], fnum(inp["D_ani"][0])]],
    "B_ext": [fnum(x) for x in inp["H_ext"]],
    "source": "tests/serial/minimization/{inp,lattice.in,SpinSTMi.dat,REF}",
}

dat = np.loadtxt(os.path.join(base, "SpinSTMi.dat"))
areal = np.asarray(vec)
frac = dat[:, :3] @ np.linalg.inv(areal)
i1 = np.rint(frac[:, 0]).astype(int) % L[0]
i2 = np.rint(frac[:, 1]).astype(int) % L[1]
cell = i1 + L[0] * i2
assert np.abs(frac[:, :2] - np.rint(frac[:, :2])).max() < 1e-6 and len(np.unique(cell)) == L[0] * L[1]
spins = np.zeros((L[0] * L[1], 3), np.int64)
spins[cell] = np.rint(dat[:, 3:6] * 1e8).astype(np.int64)
assert np.array_equal(spins[cell] / 1e8, dat[:, 3:6])  # the integers give back the parsed doubles exactly

text = open(os.path.join(base, "REF")).read()
start = float(re.search(r"starting energy\s+([-0-9.]+)", text).group(1))
energies = [float(x) for x in re.findall(r"Energy of the system \(eV/unit cell\)\s+([-0-9.]+)", text)]
torques = [float(x) for x in re.findall(r"Measured Torque:\s+([-0-9.]+)", text)]
crit = float(re.search(r"convergence criteria:\s+([0-9.]+)", text).group(1))
out = {"deck": deck, "start_energy_per_cell": start, "start_energy_digits": 6,
       "iterate_energy_per_cell": energies, "iterate_torque": torques, "convergence_criterion": crit,
       "spins": "minimization_triangular100.npz (int64 k, m = k / 1e8, site = i1 + 100 i2)"}
with open(os.path.join(HERE, "minimization_triangular100.json"), "w") as f:
    json.dump(out, f, indent=1)
np.savez_compressed(os.path.join(HERE, "minimization_triangular100.npz"), spins=spins.astype(np.int32))
print("iterates:", len(energies), "final", energies[-1], "torque", torques[-1])
