"""GNEB: the oracle's restatement of the reference's path relaxation
(find_path, GNEB/gneb_utils.f90) pinned to the reference's own GNEB test
(tests/serial/gneb/heisenberg_chain), and the host-side path tools (CPU)."""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "gneb_chain10.json")))


def chain_deck():
    from matjes_b200.deck import square_film

    g = GOLD["deck"]
    return square_film(tuple(g["L"]), Jv=g["J1"], Dv=0.0, Kv=g["K_z"], Bz=0.0, mu_s=g["mu_s"],
                       periodic=tuple(g["periodic"]))


def chain_path(seed=1):
    """Geodesic path from all +z to all -z, perturbed by 1e-3 as the reference's
    test deck asks, the end images back at the energy minima."""
    from matjes_b200.gneb import geodesic_path

    N, nim = 10, GOLD["deck"]["nim"]
    up = np.tile([0.0, 0.0, 1.0], (N, 1))
    path = geodesic_path(up, -up, nim, amp_rnd=1e-3, seed=seed)
    path[0], path[-1] = up, -up
    return np.ascontiguousarray(path)


def mz_matches(a, b, tol):
    """m_z along the chain, up to the chain's mirror symmetry (a wall may enter
    from either end)."""
    return min(np.abs(a - b).max(), np.abs(a - b[::-1]).max()) <= tol


def test_geodesic_path_and_hermite_tools():
    from matjes_b200.gneb import find_sp, geodesic_path, hermite_fit, spline_hermite_val

    up = np.tile([0.0, 0.0, 1.0], (3, 1))
    p = geodesic_path(up, -up, 5)
    # antiparallel ends: one rotation plane for every spin, pi / 4 per image
    np.testing.assert_allclose(p[2, :, 2], 0.0, atol=1e-15)
    np.testing.assert_allclose(np.linalg.norm(p, axis=2), 1.0, rtol=1e-15)
    assert np.abs(np.cross(p[1, 0], p[1, 1])).max() < 1e-15
    tilt = np.array([[math.sin(0.6), 0.0, math.cos(0.6)]] * 3)
    q = geodesic_path(up, tilt, 4)
    np.testing.assert_allclose(np.arccos(q[:, 0, 2]), [0.0, 0.2, 0.4, 0.6], atol=1e-12)
    # Hermite interpolation of a cubic is exact; its maximum found in between images
    x = np.linspace(0.0, 3.0, 7)
    f = lambda t: -(t - 1.3) ** 2 * (t + 1.0) + 5.0  # noqa: E731
    df = lambda t: -2.0 * (t - 1.3) * (t + 1.0) - (t - 1.3) ** 2  # noqa: E731
    c, xx, yy, dyy = hermite_fit(x, f(x), df(x), 31)
    np.testing.assert_allclose(yy, f(xx), rtol=1e-13)
    imax, d = find_sp(x, c)
    assert x[imax] + d == pytest.approx(1.3, abs=1e-12)
    assert spline_hermite_val(x, c, 1.3)[0] == pytest.approx(5.0, rel=1e-14)


def test_oracle_path_reproduces_the_reference_gneb_test():
    """The relaxed path of the reference's chain test: per image the reaction
    coordinate (3e-5), the energy above the first image (5e-9 eV, the barrier
    is 2.1e-3 eV) and its derivative along the path (5e-9 eV), the saddle point
    of the Hermite fit, and the spins of each image (m_z, 1e-4)."""
    from matjes_b200.gneb import saddle_point

    g = GOLD["deck"]
    mod = O.Model(chain_deck())
    path = chain_path()
    O.set_threads(1)
    try:
        rx, ene, dene, iters, fchk = O.gneb_find_path(mod, path, spring=g["spring"], dt=g["vpo_dt"],
                                                      mass=g["vpo_mass"], ftol=g["mep_ftol"], en_zero="I")
    finally:
        O.set_threads(0)
    assert fchk < g["mep_ftol"] and 10000 < iters < 200000
    ref = np.array(GOLD["en_path_out"])
    np.testing.assert_allclose(rx, ref[:, 0], rtol=0, atol=3e-5)
    np.testing.assert_allclose(ene, ref[:, 1], rtol=0, atol=5e-9)
    np.testing.assert_allclose(dene[1:-1], ref[1:-1, 2], rtol=0, atol=5e-9)
    _, (rx0, e0, de0) = saddle_point(rx, ene, dene)
    assert rx0 == pytest.approx(GOLD["ensp"][0], abs=3e-5)
    assert e0 == pytest.approx(GOLD["ensp"][1], abs=5e-9)
    for k in range(len(path)):
        assert mz_matches(path[k, :, 2], np.array(GOLD["images"][k])[:, 2], 1e-4), k


def test_oracle_climbing_image_reaches_the_saddle():
    """do_gneb_ci after the plain relaxation (GNEB_run's order): the climbing
    image is the image of highest energy, the energy's derivative along the
    path vanishes there (|dE/dx| < 1e-7 eV against 2e-3 eV of barrier), and its
    energy is the saddle point of the reference's fit to 5e-7 eV (the Hermite
    fit of 12 images overshoots the barrier by 2e-7 eV)."""
    g = GOLD["deck"]
    mod = O.Model(chain_deck())
    path = chain_path()
    O.set_threads(1)
    try:
        O.gneb_find_path(mod, path, spring=g["spring"], dt=g["vpo_dt"], mass=g["vpo_mass"], ftol=g["mep_ftol"],
                         en_zero="I")
        rx, ene, dene, iters, fchk, ci = O.gneb_find_path(mod, path, spring=g["spring"], dt=g["vpo_dt"],
                                                          mass=g["vpo_mass"], ftol=g["mep_ftol"], en_zero="I",
                                                          climb=True, return_ci=True)
    finally:
        O.set_threads(0)
    assert fchk < g["mep_ftol"] and 0 < ci < len(ene) - 1
    assert ci == int(np.argmax(ene))
    assert abs(dene[ci]) < 1e-7
    assert abs(ene[ci] - GOLD["ensp"][1]) < 5e-7


GNEB_DECK = """simulation GNEB
Periodic_log .F. .F. .F.
lattice
1.0 0.0 0.0
0.0 1.0 0.0
0.0 0.0 1.0
Nsize 10 1 1
atomtypes 1
Fe 1.0 0.0 1.0 F
atoms 1
Fe 0.0 0.0 0.0
magnetic_J
1 1 1 1.0d-3
magnetic_anisotropy
1 0.0 0.0 -0.3d-3
#spring 12.5
nim 12
do_gneb_simple .T.
mep_ftol 1.0d-8
vpo_dt 0.01
en_zero I
initpath 2
restartfile_path image-GNEB-start
momfile_i momfile_i
momfile_f momfile_f
"""


def test_gneb_keywords():
    """rw_gneb: keyword values and defaults, and initpath's settings with the
    gnebinit_* overrides; the deck builds the chain of the reference's test."""
    from matjes_b200 import reference_io as R
    from matjes_b200.deck import random_sphere

    ri = R.parse_input(GNEB_DECK)
    gi = ri.gneb
    assert ri.simulation == "GNEB" and gi.nim == 12 and gi.do_gneb and not gi.do_gneb_ci
    assert (gi.mepftol, gi.dt, gi.mass, gi.spring, gi.en_zero) == (1e-8, 0.01, 1.0, 0.5, "I")
    assert (gi.read_path, gi.read_outer, gi.min_type) == (True, True, 2)
    assert gi.restartfile_path == "image-GNEB-start" and gi.every == 10 and gi.itrmax == 2 ** 63 - 1
    for ip, want in ((1, (False, True, 0)), (3, (True, True, 1)), (7, (False, True, 1)), (-1, (False, True, 1))):
        g2 = R.parse_input(GNEB_DECK.replace("initpath 2", f"initpath {ip}")).gneb
        assert (g2.read_path, g2.read_outer, g2.min_type) == want, ip
    g3 = R.parse_input(GNEB_DECK + "gnebinit_min_type 0\ngnebinit_read_path .F.\ndo_gneb_ci .T.\n").gneb
    assert (g3.read_path, g3.min_type, g3.do_gneb_ci) == (False, 0, True)
    m = random_sphere(10, 3)
    assert np.array_equal(O.Model(ri.deck).field(m)[0], O.Model(chain_deck()).field(m)[0])


def test_gneb_files_and_saddle_configuration(tmp_path):
    """image files (3 F14.8 and two blanks per spin), en_path files (x / x0 with
    do_norm_rx 'Y'), and the spins at the saddle point on the geodesic between
    two images (find_SP_conf)."""
    from matjes_b200.gneb import saddle_configuration, write_en, write_image

    write_image(str(tmp_path / "i.dat"), np.array([[0.6, -0.8, 0.0], [0.0, 0.0, -1.0]]))
    assert (tmp_path / "i.dat").read_text() == ("    0.60000000   -0.80000000    0.00000000  \n"
                                                "    0.00000000    0.00000000   -1.00000000  \n")
    write_en(str(tmp_path / "e.out"), [1.0, 4.0], [0.5, -0.25], [0.0, 1e-3], 4.0, "Y")
    rows = [[float(v) for v in ln.split()] for ln in (tmp_path / "e.out").read_text().splitlines()]
    assert rows == [[0.25, 0.5, 0.0], [1.0, -0.25, 1e-3]]
    with pytest.raises(ValueError):
        write_en(str(tmp_path / "x.out"), [1.0], [0.0], [0.0], 1.0, "Q")
    a = np.array([[0.0, 0.0, 1.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    b = np.array([[1.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, -1.0]])
    sp = saddle_configuration(a, b, 2.0, 4.0, 3.0)
    # a quarter turn: halfway is 45 degrees in the x-z plane
    np.testing.assert_allclose(sp[0], [math.sqrt(0.5), 0.0, math.sqrt(0.5)], atol=1e-15)
    np.testing.assert_allclose(sp[1], [1.0, 0.0, 0.0], atol=1e-15)
    # antiparallel: a half turn's half about an axis perpendicular to the spin
    assert abs(sp[2, 2]) < 1e-15 and abs(np.linalg.norm(sp[2]) - 1.0) < 1e-15
