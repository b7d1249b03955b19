"""Extract the reference's GNEB test into a fixture.

Reads tests/serial/gneb/heisenberg_chain/ of the Matjes source tree (the one argument)
and writes gneb_chain10.json beside this script: the
initial and converged path energies (en_path-REF.in / en_path-REF.out: reaction
coordinate, energy above the first image, energy derivative along the path), the
saddle point of the Hermite fit (ensp_path-REF.out) and the spins of the 12
converged images (image-GNEB_<k>-REF.dat, columns x y z mx my mz |m|).  The run
(the inp, lattice.in and GNEB.in decks beside them): a chain of 10 spins, open
ends, nearest-neighbour J_1 = 1 meV, easy axis z with 0.3 meV per site, moment 1,
no field; 12 images from all +z to all -z, spring 0.5 (the default: the deck's
spring line is commented out), VPO time step 0.01 and mass 1, force tolerance
1e-8, energies relative to the initial image.
"""
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit(__doc__)
ref = sys.argv[1]
base = os.path.join(ref, "tests", "serial", "gneb", "heisenberg_chain")


def table(name):
    rows = []
    with open(os.path.join(base, name)) as f:
        for line in f:
            if line.strip():
                rows.append([float(x) for x in line.split()])
    return rows


out = {
    "en_path_in": table("en_path-REF.in"),
    "en_path_out": table("en_path-REF.out"),
    "ensp": table("ensp_path-REF.out")[0],
    "images": [[r[3:6] for r in table(f"image-GNEB_{k}-REF.dat")] for k in range(1, 13)],
    "deck": {"L": [10, 1, 1], "periodic": [0, 0, 0], "J1": 1e-3, "K_z": -0.3e-3, "mu_s": 1.0, "nim": 12,
             "spring": 0.5, "vpo_dt": 0.01, "vpo_mass": 1.0, "mep_ftol": 1e-8, "en_zero": "I",
             "source": "tests/serial/gneb/heisenberg_chain/{inp,lattice.in,GNEB.in,momfile_i,momfile_f,*-REF*}"},
}
with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "gneb_chain10.json"), "w") as f:
    json.dump(out, f, indent=1)
print("images:", len(out["images"]), "path rows:", len(out["en_path_out"]))
