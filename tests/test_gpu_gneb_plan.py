"""GNEB path relaxation on a plan (mj_gneb_path: every image's field and energy
from the plan's own field kernels) against the oracle's find_path
(GNEB/gneb_utils.f90:19-240) on lattices and terms a replica batch does not
hold: the FFT dipolar term, simple-cubic films; and on the 2D film the batch
also holds, where both device paths agree."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _path(deck, nim, seed):
    """From +z to -z along the geodesic, perturbed by 1e-2 (end images fixed)."""
    from matjes_b200.gneb import geodesic_path

    n = deck.nsites
    up = np.tile([0.0, 0.0, 1.0], (n, 1))
    path = geodesic_path(up, -up, nim, amp_rnd=1e-2, seed=seed)
    path[0], path[-1] = up, -up
    return np.ascontiguousarray(path)


def _decks():
    from matjes_b200.deck import Deck, square_areal, square_film

    film = dict(Jv=1e-3, Dv=0.4e-3, Kv=-0.2e-3, Bz=0.3, mu_s=2.0, a=0.25, med_z=-0.3, periodic=(1, 1, 0))
    return {
        "dipolar_film_8x8x2": square_film((8, 8, 2), dip=True, **film),
        "cubic_film_6x6x3": square_film((6, 6, 3), **film),
        "two_atom_cell_ell_6x5": Deck(L=(6, 5, 1), periodic=(1, 1, 0), areal=square_areal(),
                                      atoms=[((0, 0, 0), 1, 2.0), ((0.5, 0.5, 0), 1, 1.5), ((0.5, 0.0, -0.5), 2, 0.0)],
                                      J=[(1, 1, 1, 1e-3), (1, 1, 2, 0.4e-3)], D=[(1, 1, 2, 1, 0.2e-3)],
                                      K=[(1, (0, 0, 1), -0.1e-3)], B_ext=(0, 0, 0.7)),
    }


@pytest.mark.parametrize("name", ["dipolar_film_8x8x2", "cubic_film_6x6x3"])
@pytest.mark.parametrize("climb", [False, True])
def test_plan_path_follows_the_oracle(name, climb):
    """200 iterations (ftol 0: no early stop), plain and climbing: the images,
    rx, ene and dene equal the oracle's to the rounding of the summation order
    (1e-10 relative; a 1e-13 change of these paths' start stays below 1e-12
    through 200 oracle iterations, so nothing amplifies the rounding)."""
    from matjes_b200.gneb import GNEBInput, PlanPath, find_path

    deck = _decks()[name]
    path = _path(deck, 6, seed=5)
    inp = GNEBInput(spring=0.3, dt=0.02, mass=1.0, mepftol=0.0, mepftol_ci=0.0, itrmax=200, en_zero="I")
    res = find_path(deck, path, inp, climb=climb)
    op = path.copy()
    orx, oene, odene, oit, ofc, oci = O.gneb_find_path(O.Model(deck), op, spring=0.3, dt=0.02, mass=1.0, ftol=0.0,
                                                       itrmax=200, en_zero="I", climb=climb, return_ci=True)
    assert res.iterations == oit == 200 and res.ci == oci
    assert np.abs(res.images - op).max() < 1e-10
    np.testing.assert_allclose(res.rx, orx, rtol=1e-10)
    assert np.abs(res.ene - oene).max() <= 1e-10 * np.abs(oene).max()
    assert np.abs(res.dene - odene).max() <= 1e-10 * np.abs(odene).max()
    assert res.max_force == pytest.approx(ofc, rel=1e-9)
    # the end images do not move
    np.testing.assert_array_equal(res.images[0], path[0])
    np.testing.assert_array_equal(res.images[-1], path[-1])
    # these decks are held on a plan, not as replicas
    from matjes_b200.gneb import path_holder

    assert isinstance(path_holder(deck, path), PlanPath)


def test_plan_and_replica_paths_agree():
    """The 2D DMI film both holders take: the plan's relaxation (tiled field
    kernels per image) and the batch's (the fused GNEB field pass) end at the
    same path after 200 iterations (1e-10; this path's own sensitivity grows a
    1e-13 change to 1e-7 between iterations 280 and 300, so the comparison stops
    well before), and stop within two iterations of each other under a
    tolerance that the path reaches after about 220."""
    from matjes_b200 import Hamiltonian
    from matjes_b200.deck import square_film
    from matjes_b200.gneb import GNEBInput, find_path, find_path_plan

    deck = square_film((8, 6, 1), Jv=1e-3, Dv=0.4e-3, Kv=-0.2e-3, Bz=0.3, mu_s=2.0, periodic=(1, 1, 0))
    path = _path(deck, 6, seed=5)
    inp = GNEBInput(spring=0.3, dt=0.02, mass=1.0, mepftol=0.0, itrmax=200, en_zero="F")
    a = find_path(deck, path, inp)
    b = find_path_plan(Hamiltonian(deck), path, inp)
    assert a.iterations == b.iterations == 200
    assert np.abs(a.images - b.images).max() < 1e-10
    np.testing.assert_allclose(a.rx, b.rx, rtol=1e-10)
    assert np.abs(a.ene - b.ene).max() <= 1e-10 * np.abs(a.ene).max()
    inp = GNEBInput(spring=0.3, dt=0.02, mass=1.0, mepftol=2e-4, itrmax=100000, en_zero="I")
    a = find_path(deck, path, inp)
    b = find_path_plan(Hamiltonian(deck), path, inp)
    assert a.max_force < 2e-4 and b.max_force < 2e-4
    assert abs(a.iterations - b.iterations) <= 2
    assert np.abs(a.images - b.images).max() < 1e-6


def test_plan_and_replica_paths_agree_with_many_images_and_tma_staging():
    """14 images of a 64 x 64 DMI film: more images than the plan path's 8
    forked streams (several images queued on one stream) and a lattice whose
    interior tiles the plan's field kernels stage by TMA (the default).  After 60
    iterations the plan's path equals the batch's (the fused GNEB field pass) to
    1e-10, reaction coordinates and energies included."""
    from matjes_b200 import Hamiltonian
    from matjes_b200._abi import lib
    from matjes_b200.deck import square_film
    from matjes_b200.gneb import GNEBInput, find_path, find_path_plan

    deck = square_film((64, 64, 1), Jv=1e-3, Dv=0.4e-3, Kv=-0.2e-3, Bz=0.3, mu_s=2.0, periodic=(1, 1, 0))
    path = _path(deck, 14, seed=6)
    inp = GNEBInput(spring=0.3, dt=0.02, mass=1.0, mepftol=0.0, itrmax=60, en_zero="I")
    a = find_path(deck, path, inp)
    ham = Hamiltonian(deck)
    variant, shape = C.c_int32(), C.c_int32()
    assert lib.mj_plan_get_variant(ham.plan, C.byref(variant), C.byref(shape)) == 0
    assert variant.value >= 0 and shape.value != 0  # tiled kernels, TMA staging on by default
    b = find_path_plan(ham, path, inp)
    assert a.iterations == b.iterations == 60
    assert np.abs(a.images - b.images).max() < 1e-10
    np.testing.assert_allclose(a.rx, b.rx, rtol=1e-10)
    assert np.abs(a.ene - b.ene).max() <= 1e-10 * np.abs(a.ene).max()


def test_plan_path_arguments_are_checked():
    import torch

    from matjes_b200 import Hamiltonian
    from matjes_b200._abi import MJ_ERR_ARG, MJ_ERR_UNSUPPORTED, GnebParams, lib

    deck = _decks()["cubic_film_6x6x3"]
    ham = Hamiltonian(deck)
    m = torch.zeros((3, 3, ham.N), dtype=torch.float64, device="cuda:0")
    m[:, 2] = 1.0
    rx, ene, dene = np.zeros(3), np.zeros(3), np.zeros(3)
    p = lambda a: a.ctypes.data  # noqa: E731
    gp = lambda dt, ez: C.byref(GnebParams(0.5, dt, 1.0, 1e-3, 10, ord(ez), 0))  # noqa: E731
    d = C.c_void_p(m.data_ptr())
    assert lib.mj_gneb_path(ham.plan, d, 2, gp(0.01, "I"), p(rx), p(ene), p(dene), None, None, None, None) == MJ_ERR_ARG
    assert lib.mj_gneb_path(ham.plan, d, 3, gp(0.01, "X"), p(rx), p(ene), p(dene), None, None, None, None) == MJ_ERR_ARG
    assert lib.mj_gneb_path(ham.plan, d, 3, gp(-0.01, "I"), p(rx), p(ene), p(dene), None, None, None,
                            None) == MJ_ERR_ARG
    assert lib.mj_gneb_path(ham.plan, None, 3, gp(0.01, "I"), p(rx), p(ene), p(dene), None, None, None,
                            None) == MJ_ERR_ARG
    assert lib.mj_gneb_path(None, d, 3, gp(0.01, "I"), p(rx), p(ene), p(dene), None, None, None, None) == MJ_ERR_ARG
    with pytest.raises(ValueError):
        from matjes_b200.gneb import PlanPath

        PlanPath(ham, np.zeros((3, ham.N + 1, 3)))
    # two magnetic atoms per cell: refused, as the reference's find_path stops
    two = Hamiltonian(_decks()["two_atom_cell_ell_6x5"])
    m2 = torch.zeros((3, 3, two.N), dtype=torch.float64, device="cuda:0")
    assert lib.mj_gneb_path(two.plan, C.c_void_p(m2.data_ptr()), 3, gp(0.01, "I"), p(rx), p(ene), p(dene), None,
                            None, None, None) == MJ_ERR_UNSUPPORTED
