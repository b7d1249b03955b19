"""Extract the reference's isolated-spin-precession golden logs into a fixture.

Reads tests/serial/isolated_spin_precession/{Euler/REF,Heun/EM.dat} of the
Matjes source tree (the one argument) and writes
isolated_spin_precession.json beside this script: per step the columns
time (fs), E_av (eV), |M|, Mx, My, Mz of the 4x4 ferromagnet in B = 10 T z,
m0 = x, dt = 1 fs, alpha = 0, mu_s = 1, J_1 = 1e-6 eV (the decks beside the logs).
"""
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit(__doc__)
ref = sys.argv[1]
base = os.path.join(ref, "tests", "serial", "isolated_spin_precession")
out = {}
for name, fn in (("euler", "Euler/REF"), ("heun", "Heun/EM.dat")):
    rows = []
    with open(os.path.join(base, fn)) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            v = [float(x) for x in line.split()]
            rows.append(v[:6])
    out[name] = {"columns": ["time_fs", "E_av_eV", "M", "Mx", "My", "Mz"], "rows": rows}
out["deck"] = {"L": [4, 4, 1], "B_ext": [0.0, 0.0, 10.0], "J1": 1e-6, "mu_s": 1.0, "timestep_fs": 1.0,
               "alpha": 0.0, "m0": [1.0, 0.0, 0.0], "steps": 50,
               "source": "tests/serial/isolated_spin_precession/{Euler/REF,Heun/EM.dat} and the inp/dyna.in decks"}
with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "isolated_spin_precession.json"), "w") as f:
    json.dump(out, f, indent=1)
print("rows:", len(out["euler"]["rows"]), len(out["heun"]["rows"]))
