"""Extract the reference's parallel-tempering Monte Carlo golden log into a fixture.

Reads tests/serial/PTMC/EM.dat of the Matjes source tree (the one argument)
and writes ptmc_ising_square20.json beside this script: per
temperature the columns T (K), E_av (eV per site), E_err (per-site sample
standard deviation of the measured energies), C, M (norm of the averaged
summed spins per site), Mx, My, Mz; plus the text tokens of three rows for the
(E20.10E3) number format.  The run (the inp and lattice.in decks beside the
log): a 20 x 20 square lattice, periodic in plane, nearest-neighbour J_1 =
0.5e-3 eV per directed pair (c_Ji = -1), on-site term +5e-7 eV per site along
z (constant under Ising moves), no field, Ising sampling from the +z state, 40
temperatures from 1 to 61 K.  The log holds 100 measurements per temperature:
its C column equals E_err^2 N (n - 1) / n / kT^2 with n = 100 on every row.
"""
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit(__doc__)
ref = sys.argv[1]
path = os.path.join(ref, "tests", "serial", "PTMC", "EM.dat")
rows, tokens = [], []
with open(path) as f:
    for line in f:
        if line.startswith("#") or not line.strip():
            continue
        t = line.split()
        v = [float(x) for x in t]
        if v[0] <= 0.0:  # unused trailing rows of the log
            continue
        rows.append(v[:8])
        if len(tokens) < 3 or len(rows) in (16, 40):
            tokens.append(t)
out = {
    "columns": ["T_K", "E_av_eV", "E_err_eV", "C", "M", "Mx", "My", "Mz"],
    "rows": rows,
    "tokens": tokens,
    "deck": {"L": [20, 20, 1], "periodic": [1, 1, 0], "J1": 0.5e-3, "K_z": 5e-7, "mu_s": 3.0, "B_ext": [0, 0, 0],
             "sampling": "ising", "m0": [0.0, 0.0, 1.0], "T_ini": 1.0, "T_fin": 61.0, "n_Tsteps": 40,
             "measurements": 100, "source": "tests/serial/PTMC/{EM.dat,inp,lattice.in}"},
}
with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "ptmc_ising_square20.json"), "w") as f:
    json.dump(out, f, indent=1)
print("rows:", len(rows))
