"""The reference's input deck and file formats (matjes_b200.reference_io), CPU."""
import numpy as np
import pytest

from oracle import oracle as O

DECK = """# square film: J, interfacial DMI from a mediator below the plaquette centre
simulation magnet-dynamics
Periodic_log .T. .T. .F.
alat 1.0d0 1.0d0 1.0d0
lattice
2.0 0.0 0.0
0.0 1.0 0.0
0.0 0.0 1.0
Nsize 24 20 1
atomtypes 2
Fe 2.0 0.0 1.0 F
Ir 0.0 0.0 1.0 F
atoms 2
Fe 0.0 0.0 0.0
Ir 1 1 -1 2
magnetic_J
# t1 t2 shell J
1 1 1 1.0d-3
1 1 2 0.0
magnetic_D
1 1 2 1 0.3d-3
magnetic_anisotropy
1 0.0 0.0 -0.1d-3
H_ext 0.0 0.0 0.5
timestep 0.1
duration 30
damping 0.3
Efreq 10
integration 3
Tini 0.0d0
masse 2.0
convergence_criteria 1.0d-7
"""


def test_input_deck_builds_the_same_model_as_the_deck_api():
    from matjes_b200 import reference_io as R
    from matjes_b200.deck import random_sphere, square_film

    ri = R.parse_input(DECK)
    d = ri.deck
    assert d.L == (24, 20, 1) and d.periodic == (1, 1, 0)
    # the lattice row of length 2 is normalised with its length folded into alat
    np.testing.assert_allclose(d.areal, np.diag([2.0, 1.0, 1.0]))
    assert d.atoms == [((0.0, 0.0, 0.0), 1, 2.0), ((0.5, 0.5, -0.5), 2, 0.0)]
    assert d.J == [(1, 1, 1, 1e-3)]          # the zero entry is dropped
    assert d.D == [(1, 1, 2, 1, 0.3e-3)]
    # the 3-real anisotropy form: magnitude |k| with the sign of the last non-zero component
    assert d.K == [(1, (0.0, 0.0, -0.1e-3), -0.1e-3)]
    assert d.B_ext == (0.0, 0.0, 0.5)
    assert (ri.dynamics.integration, ri.dynamics.duration, ri.dynamics.Efreq) == (3, 30, 10)
    assert ri.dynamics.damping == 0.3 and ri.minimize.mass == 2.0 and ri.minimize.conv_torque == 1e-7
    # the same couplings as the deck built through the API (lattice constant 2 along x)
    ref = square_film((24, 20, 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.5)
    ref.areal = np.diag([2.0, 1.0, 1.0])
    m = random_sphere(d.nsites, 5)
    Ba, _ = O.Model(d).field(m)
    Bb, _ = O.Model(ref).field(m)
    assert np.array_equal(Ba, Bb)


def test_anisotropy_four_real_form_and_rotation():
    from matjes_b200 import reference_io as R

    text = DECK.replace("1 0.0 0.0 -0.1d-3", "1 0.0 0.0 1.0 -0.1d-3") + "rotate_lattice 0.5 0.0 0.0\n"
    d = R.parse_input(text).deck
    assert d.K == [(1, (0.0, 0.0, 1.0), -0.1e-3)]
    # rows times the Z-X-Z matrix (net = matmul(net, rot_mat)): 0.5 pi about z takes x to -y
    np.testing.assert_allclose(d.areal[0], [0.0, -2.0, 0.0], atol=1e-15)


def test_fortran_e_format_known_answers():
    from matjes_b200.reference_io import fortran_e

    assert fortran_e(1.0, 20, 12, 3) == " 0.100000000000E+001"
    assert fortran_e(-2.5e-10, 20, 12, 3) == "-0.250000000000E-009"
    assert fortran_e(0.0, 24, 16) == "  0.0000000000000000E+00"
    assert fortran_e(0.99999999999999999, 24, 16) == "  0.1000000000000000E+01"
    assert fortran_e(-1e120, 24, 16) == " -0.1000000000000000+121"


def test_order_files_round_trip_and_size_checks(tmp_path):
    from matjes_b200 import reference_io as R
    from matjes_b200.deck import random_sphere

    m = random_sphere(37, 9)
    p = tmp_path / "magnetic_final.dat"
    R.write_order_file(str(p), m)
    lines = p.read_text().splitlines()
    assert len(lines) == 37 and all(len(ln) == 3 * 24 + 2 for ln in lines)
    back = R.read_order_file(str(p), 37)
    assert np.abs(back - m).max() <= 1e-16 * 4
    # the reference reads list-directed: any layout, Fortran exponents
    q = tmp_path / "magnetic_init.dat"
    q.write_text("0.0d0 0.0 1.0\n 1.0 0.0 0.0 0.0 1.0d0\n0.0\n")
    np.testing.assert_array_equal(R.read_order_file(str(q), 3), [[0, 0, 1], [1, 0, 0], [0, 1, 0]])
    with pytest.raises(ValueError, match="end of file"):
        R.read_order_file(str(q), 4)
    with pytest.raises(ValueError, match="further entries"):
        R.read_order_file(str(q), 2)
    b = tmp_path / "Beff_3.dat"
    R.write_beff(str(b), m[:4])
    assert all(len(ln) == 3 * 22 for ln in b.read_text().splitlines())


def test_em_dat_rows():
    from matjes_b200 import reference_io as R

    assert R.em_header().startswith("# 1:step  2:real_time (fs)  3:E_av (eV)")
    row = R.em_line(11, 1.1, -2.25, [0.0, 0.6, 0.8], 10.0, 9.5, [0.0, 0.0, 1.0])
    assert row.endswith("\n") and len(row.rstrip("\n")) == 12 + 17 * 22 + 20
    vals = [float(x) for x in row.split()]
    assert vals[0] == 11 and vals[2] == -2.25 and vals[3] == pytest.approx(1.0, rel=1e-12)
    assert vals[14:19] == [10.0, 9.5, 0.0, 0.0, 1.0]
    # without calc_topo the topology columns hold the reference's placeholder values
    assert vals[11] == pytest.approx(2 * 1.2345789e98, rel=1e-9)


MC_DECK = """simulation metropolis
Periodic_log .T. .T. .F.
lattice
1.0 0.0 0.0
0.0 1.0 0.0
0.0 0.0 1.0
Nsize 20 20 1
atomtypes 1
Fe 3.0 0.0 1.0 F
atoms 1
Fe 0.0 0.0 0.0
magnetic_J
1 1 1 0.5d-3
magnetic_anisotropy
1 0.0 0.0 1.0 5.0d-7
Tini 10.0
Tfin 30.0
n_Tsteps 3
n_relaxation 50
T_relax 2
T_auto 3
Total_MC_Steps 400
cone 0.8
ising .T.
"""


def test_monte_carlo_keywords():
    from matjes_b200 import reference_io as R

    ri = R.parse_input(MC_DECK)
    mc = ri.monte_carlo
    assert ri.simulation == "metropolis" and mc.sampling == "ising"
    assert (mc.n_Tsteps, mc.N_relaxation, mc.T_relax, mc.T_auto, mc.Total_MC_Steps) == (3, 50, 2, 3, 400)
    assert mc.cone == 0.8 and mc.n_sizerelax == 1
    assert (ri.dynamics.Tini, ri.dynamics.Tfin) == (10.0, 30.0)
    # rw_MC: one method exactly; get_bool needs the value after the keyword
    assert R.parse_input(MC_DECK.replace("ising .T.", "ising .F.")).monte_carlo is None
    with pytest.raises(ValueError, match="more than one"):
        R.parse_input(MC_DECK + "sphere_samp .T.\n")
    with pytest.raises(ValueError, match="expected 1 values"):
        R.parse_input(MC_DECK.replace("ising .T.", "ising"))
