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
