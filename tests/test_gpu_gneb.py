"""GNEB path relaxation on the device (mj_batch_gneb_path, the images held as
the replicas of a batch) against the oracle's find_path (GNEB/gneb_utils.f90:
19-240) and the reference's own chain test (tests/serial/gneb/heisenberg_chain)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "gneb_chain10.json")))


def _chain():
    from test_gneb_oracle import chain_deck, chain_path

    return chain_deck(), chain_path()


def _film_path(nim=6, L=(8, 6), seed=5, fixed_ends=True):
    """A DMI film with a perpendicular field; the path from +z to -z, perturbed
    by 1e-2 so that every image leaves the geodesic (the end images too unless
    fixed_ends)."""
    from matjes_b200.deck import square_film
    from matjes_b200.gneb import geodesic_path

    deck = square_film((L[0], L[1], 1), Jv=1e-3, Dv=0.4e-3, Kv=-0.2e-3, Bz=0.3, mu_s=2.0, periodic=(1, 1, 0))
    n = L[0] * L[1]
    up = np.tile([0.0, 0.0, 1.0], (n, 1))
    path = geodesic_path(up, -up, nim, amp_rnd=1e-2, seed=seed)
    if fixed_ends:
        path[0], path[-1] = up, -up
    return deck, np.ascontiguousarray(path)


def test_device_path_reproduces_the_reference_gneb_test():
    """The relaxed chain path: rx (3e-5), energies above image 0 (5e-9 eV; the
    barrier is 2.1e-3 eV), the derivative along the path (5e-9 eV), the saddle
    point of the Hermite fit and every image's m_z (1e-4, up to the mirror)."""
    from matjes_b200.gneb import GNEBInput, find_path, saddle_point
    from test_gneb_oracle import mz_matches

    g = GOLD["deck"]
    deck, path = _chain()
    inp = GNEBInput(nim=g["nim"], spring=g["spring"], dt=g["vpo_dt"], mass=g["vpo_mass"], mepftol=g["mep_ftol"],
                    en_zero="I")
    res = find_path(deck, path, inp)
    out, rx, ene, dene, iters, fchk = res.images, res.rx, res.ene, res.dene, res.iterations, res.max_force
    assert fchk < g["mep_ftol"] and 10000 < iters < 200000
    ref = np.array(GOLD["en_path_out"])
    np.testing.assert_allclose(rx, ref[:, 0], rtol=0, atol=3e-5)
    np.testing.assert_allclose(ene, ref[:, 1], rtol=0, atol=5e-9)
    np.testing.assert_allclose(dene[1:-1], ref[1:-1, 2], rtol=0, atol=5e-9)
    _, (rx0, e0, _) = saddle_point(rx, ene, dene)
    assert rx0 == pytest.approx(GOLD["ensp"][0], abs=3e-5)
    assert e0 == pytest.approx(GOLD["ensp"][1], abs=5e-9)
    for k in range(len(out)):
        assert mz_matches(out[k, :, 2], np.array(GOLD["images"][k])[:, 2], 1e-4), k
    # the end images do not move
    np.testing.assert_array_equal(out[0], path[0])
    np.testing.assert_array_equal(out[-1], path[-1])
    # the oracle's relaxation of the same path ends at the same images (both stop
    # at max |F| < 1e-8, a few iterations apart: 1e-9 eV on the energies)
    op = path.copy()
    O.set_threads(1)
    try:
        orx, oene, odene, oit, _ = O.gneb_find_path(O.Model(deck), op, spring=g["spring"], dt=g["vpo_dt"],
                                                    mass=g["vpo_mass"], ftol=g["mep_ftol"], en_zero="I")
    finally:
        O.set_threads(0)
    assert abs(iters - oit) <= max(50, oit // 100)
    np.testing.assert_allclose(ene, oene, rtol=0, atol=1e-9)
    assert np.abs(out - op).max() < 1e-6


@pytest.mark.parametrize("en_zero", ["I", "F", "N"])
def test_device_iterations_follow_the_oracle(en_zero):
    """200 iterations of a 2D film path (ftol 0: no early stop): the images, rx,
    ene and dene of the device run equal the oracle's to the rounding of the
    summation order (1e-10 relative).  Up to iteration 280 the oracle itself
    carries a 1e-13 change of the initial path unamplified; between iterations
    280 and 300 the same change grows to 1e-7 (the relaxation's own
    sensitivity, not the device's), so the comparison stops well before."""
    from matjes_b200.gneb import GNEBInput, find_path

    deck, path = _film_path()
    inp = GNEBInput(spring=0.3, dt=0.02, mass=1.0, mepftol=0.0, itrmax=200, en_zero=en_zero)
    res = find_path(deck, path, inp)
    out, rx, ene, dene, iters, fchk = res.images, res.rx, res.ene, res.dene, res.iterations, res.max_force
    op = path.copy()
    orx, oene, odene, oit, ofc = O.gneb_find_path(O.Model(deck), op, spring=0.3, dt=0.02, mass=1.0, ftol=0.0,
                                                  itrmax=200, en_zero=en_zero)
    assert iters == oit == 200
    assert np.abs(out - op).max() < 1e-10
    np.testing.assert_allclose(rx, orx, rtol=1e-10, atol=1e-12)
    scale = np.abs(oene).max() + 1e-3
    assert np.abs(ene - oene).max() <= 1e-10 * scale
    assert np.abs(dene - odene).max() <= 1e-10 * (np.abs(odene).max() + 1e-6)
    assert fchk == pytest.approx(ofc, rel=1e-9)


def test_triangular_three_shell_path_follows_the_oracle():
    """The GNEB field pass on the triangular three-shell stencil (J1..J3 + D1 + K
    + Bz = 1 T, 24 x 20, 7 images): 120 iterations, plain and climbing, against
    the oracle's (1e-10; the oracle carries a 1e-13 change of this path's start
    unamplified through 150 iterations)."""
    from matjes_b200.deck import triangular
    from matjes_b200.gneb import GNEBInput, find_path, geodesic_path

    deck = triangular((24, 20))
    n = 24 * 20
    up = np.tile([0.0, 0.0, 1.0], (n, 1))
    path = geodesic_path(up, -up, 7, amp_rnd=1e-2, seed=4)
    path[0], path[-1] = up, -up
    path = np.ascontiguousarray(path)
    for climb in (False, True):
        inp = GNEBInput(spring=0.3, dt=0.02, mass=1.0, mepftol=0.0, mepftol_ci=0.0, itrmax=120, en_zero="F")
        res = find_path(deck, path, inp, climb=climb)
        op = path.copy()
        orx, oene, odene, oit, ofc, oci = O.gneb_find_path(O.Model(deck), op, spring=0.3, dt=0.02, mass=1.0,
                                                           ftol=0.0, itrmax=120, en_zero="F", climb=climb,
                                                           return_ci=True)
        assert res.iterations == oit == 120 and res.ci == oci
        assert np.abs(res.images - op).max() < 1e-10
        np.testing.assert_allclose(res.rx, orx, rtol=1e-10)
        assert np.abs(res.ene - oene).max() <= 1e-10 * np.abs(oene).max()
        assert np.abs(res.dene - odene).max() <= 1e-10 * np.abs(odene).max()


def test_large_path_iterations_follow_the_oracle():
    """A path of 12 images of 160 x 160 (307,200 sites: the kernels then take four
    sites per thread): 20 iterations against the oracle's (1e-10)."""
    from matjes_b200.gneb import GNEBInput, find_path

    deck, path = _film_path(nim=12, L=(160, 160), seed=3)
    inp = GNEBInput(spring=0.3, dt=0.02, mass=1.0, mepftol=0.0, itrmax=20, en_zero="I")
    res = find_path(deck, path, inp)
    out, rx, ene, dene, iters, fchk = res.images, res.rx, res.ene, res.dene, res.iterations, res.max_force
    op = path.copy()
    orx, oene, odene, oit, ofc = O.gneb_find_path(O.Model(deck), op, spring=0.3, dt=0.02, mass=1.0, ftol=0.0,
                                                  itrmax=20, en_zero="I")
    assert iters == oit == 20
    assert np.abs(out - op).max() < 1e-10
    np.testing.assert_allclose(rx, orx, rtol=1e-10)
    assert np.abs(ene - oene).max() <= 1e-10 * np.abs(oene).max()
    assert np.abs(dene - odene).max() <= 1e-10 * np.abs(odene).max()
    assert fchk == pytest.approx(ofc, rel=1e-9)


def test_no_iteration_reports_the_initial_path():
    """itrmax 0: nothing moves; rx, ene and dene (the end images' from their
    projected fields) and max |F| are those of the initial path, as the oracle's."""
    from matjes_b200.gneb import GNEBInput, find_path

    deck, path = _film_path(nim=4, seed=9, fixed_ends=False)
    res = find_path(deck, path, GNEBInput(itrmax=0, en_zero="N"))
    out, rx, ene, dene, iters, fchk = res.images, res.rx, res.ene, res.dene, res.iterations, res.max_force
    op = path.copy()
    orx, oene, odene, oit, ofc = O.gneb_find_path(O.Model(deck), op, itrmax=0, en_zero="N")
    assert iters == oit == 0
    np.testing.assert_array_equal(out, path)
    np.testing.assert_allclose(rx, orx, rtol=1e-12)
    assert np.abs(ene - oene).max() <= 1e-12 * np.abs(oene).max()
    assert np.abs(dene - odene).max() <= 1e-11 * np.abs(odene).max()
    assert abs(dene[0]) > 0.0 and abs(dene[-1]) > 0.0
    assert fchk == pytest.approx(ofc, rel=1e-12)


def test_path_arguments_are_checked():
    import matjes_b200 as mj
    import ctypes as C

    from matjes_b200._abi import MJ_ERR_ARG, MJ_ERR_UNSUPPORTED, GnebParams, lib

    deck, path = _film_path(nim=3)
    n = path.shape[1]
    two = mj.ReplicaBatch(deck, [deck.L[:2]] * 2, np.zeros((2, 3)), [0.0] * 2)
    two.upload(np.concatenate(path[:2]))
    with pytest.raises(mj.MatjesError):
        two.gneb_path()
    three = mj.ReplicaBatch(deck, [deck.L[:2]] * 3, np.zeros((3, 3)), [0.0] * 3)
    three.upload(path.reshape(3 * n, 3))
    with pytest.raises(ValueError):
        three.gneb_path(en_zero="X")
    rx, ene, dene = np.zeros(3), np.zeros(3), np.zeros(3)
    p = lambda a: a.ctypes.data  # noqa: E731
    gp = lambda dt, ez: C.byref(GnebParams(0.5, dt, 1.0, 1e-3, 10, ord(ez), 0))  # noqa: E731
    assert lib.mj_batch_gneb_path(three.handle, gp(0.01, "X"), p(rx), p(ene), p(dene), None, None,
                                  None) == MJ_ERR_ARG
    assert lib.mj_batch_gneb_path(three.handle, gp(-0.01, "I"), p(rx), p(ene), p(dene), None, None,
                                  None) == MJ_ERR_ARG
    assert lib.mj_batch_gneb_path(three.handle, None, p(rx), p(ene), p(dene), None, None, None) == MJ_ERR_ARG
    mixed = mj.ReplicaBatch(deck, [deck.L[:2], (4, 6), deck.L[:2]], np.zeros((3, 3)), [0.0] * 3)
    assert lib.mj_batch_gneb_path(mixed.handle, gp(0.01, "I"), p(rx), p(ene), p(dene), None, None,
                                  None) == MJ_ERR_UNSUPPORTED


def test_device_climbing_image_follows_the_oracle():
    """The climbing-image relaxation (do_gneb_ci): 200 iterations of a 2D film
    path against the oracle's (1e-10), the same climbing image."""
    from matjes_b200.gneb import GNEBInput, find_path

    deck, path = _film_path()
    inp = GNEBInput(spring=0.3, dt=0.02, mass=1.0, mepftol_ci=0.0, itrmax=200, en_zero="I")
    res = find_path(deck, path, inp, climb=True)
    op = path.copy()
    orx, oene, odene, oit, ofc, oci = O.gneb_find_path(O.Model(deck), op, spring=0.3, dt=0.02, mass=1.0, ftol=0.0,
                                                       itrmax=200, en_zero="I", climb=True, return_ci=True)
    assert res.iterations == oit == 200 and res.ci == oci and 0 < oci < len(path) - 1
    assert np.abs(res.images - op).max() < 1e-10
    np.testing.assert_allclose(res.rx, orx, rtol=1e-10, atol=1e-12)
    assert np.abs(res.ene - oene).max() <= 1e-10 * np.abs(oene).max()
    assert np.abs(res.dene - odene).max() <= 1e-10 * np.abs(odene).max()
    # without climbing the same path goes elsewhere
    plain = find_path(deck, path, inp)
    assert plain.ci == -1 and np.abs(plain.images - res.images).max() > 1e-6


def test_reference_deck_directory_runs_the_gneb(tmp_path):
    """run_gneb on an input directory holding the reference's chain test in
    the current input format (the path read from image-GNEB-start_<k>.dat, the
    end states from momfile_i / momfile_f, minimised by `minimize`): en_path.out,
    ensp_path.out and the images against the reference's own outputs; then with
    do_gneb_ci the climbing image against the oracle's."""
    from matjes_b200 import reference_io as R
    from test_gneb_oracle import GNEB_DECK, mz_matches

    g = GOLD["deck"]
    _, path = _chain()
    for k, img in enumerate(path, start=1):
        R.write_order_file(str(tmp_path / f"image-GNEB-start_{k}.dat"), img)
    R.write_order_file(str(tmp_path / "momfile_i"), path[0])
    R.write_order_file(str(tmp_path / "momfile_f"), path[-1])
    (tmp_path / "input").write_text(GNEB_DECK)
    out = R.run_gneb(str(tmp_path))
    rows = np.array([[float(v) for v in ln.split()] for ln in (tmp_path / "en_path.out").read_text().splitlines()])
    ref = np.array(GOLD["en_path_out"])
    np.testing.assert_allclose(rows[:, 0], ref[:, 0], rtol=0, atol=3e-5)
    np.testing.assert_allclose(rows[:, 1], ref[:, 1], rtol=0, atol=5e-9)
    np.testing.assert_allclose(rows[1:-1, 2], ref[1:-1, 2], rtol=0, atol=5e-9)
    sp = [float(v) for v in (tmp_path / "ensp_path.out").read_text().split()]
    assert sp[0] == pytest.approx(GOLD["ensp"][0], abs=3e-5) and sp[1] == pytest.approx(GOLD["ensp"][1], abs=5e-9)
    assert len((tmp_path / "enfit_path.out").read_text().splitlines()) == 500
    assert len((tmp_path / "en_path.in").read_text().splitlines()) == 12
    for k in range(1, 13):
        img = np.loadtxt(str(tmp_path / f"image-GNEB_{k}.dat"))
        assert img.shape == (10, 3)
        assert mz_matches(img[:, 2], np.array(GOLD["images"][k - 1])[:, 2], 1e-4), k
    saddle = np.loadtxt(str(tmp_path / "image-GNEB-saddlepoint.dat"))
    assert saddle.shape == (10, 3) and np.abs(np.linalg.norm(saddle, axis=1) - 1.0).max() < 1e-7
    # the climbing image after the plain relaxation, against the oracle's
    (tmp_path / "input").write_text(GNEB_DECK + "do_gneb_ci .T.\nmep_ftol_ci 1.0d-8\n")
    ci_out = R.run_gneb(str(tmp_path))
    run = ci_out["runs"][-1]
    op = out["images"].copy()
    orx, oene, odene, oit, ofc, oci = O.gneb_find_path(O.Model(R.parse_input(GNEB_DECK).deck), op.copy(),
                                                       spring=g["spring"], dt=g["vpo_dt"], mass=g["vpo_mass"],
                                                       ftol=1e-8, en_zero="I", climb=True, return_ci=True)
    assert run.ci == oci and ci_out["saddle"][0] == pytest.approx(run.rx[run.ci], abs=0)
    assert abs(run.ene[run.ci] - oene[oci]) < 1e-9 and abs(run.dene[run.ci]) < 1e-7
