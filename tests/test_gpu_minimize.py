"""Energy minimisation on the device (mj_minimize, mj_minimize_infdamp) against
the oracle's restatements of solvers/minimize.F90.

The velocity-projection driver follows minimize_run step by step, so the GPU
and oracle iterates agree to rounding (the global sums V.F and |F|^2 are
added in different orders); the infinite-damping sweep is compared with the
oracle run in the same colour order, and its minimum with the one the
reference's site order reaches."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _run_gpu(deck, m0, **kw):
    import torch

    import matjes_b200 as mj

    ham = mj.Hamiltonian(deck)
    m = torch.tensor(m0.T.copy(), device="cuda")
    out = mj.minimize(ham, m, **kw)
    torch.cuda.synchronize()
    return out, m.cpu().numpy().T.copy()


@pytest.mark.parametrize("name", ["square", "film_dipolar"])
def test_velocity_projection_follows_the_reference_iterates(name):
    import matjes_b200 as mj

    if name == "square":
        deck = mj.square_film((32, 24, 1), Jv=1e-3, Dv=0.3e-3, Kv=-0.1e-3, Bz=0.5)
    else:
        deck = mj.square_film((12, 12, 3), Jv=1e-3, Dv=0.15e-3, Kv=-0.02e-3, Bz=0.2, a=0.25, med_z=-0.3, dip=True)
    m0 = mj.random_sphere(deck.nsites, 21)
    # a fixed number of iterations (criterion out of reach), then to convergence
    (it, mt), m = _run_gpu(deck, m0, method="vpo", timestep=0.1, mass=1.0, conv_torque=1e-30, max_iter=200,
                           check_every=50)
    mo = m0.copy()
    ito, mto = O.minimize_vpo(O.Model(deck), mo, 0.1, 1.0, 1e-30, 200)
    assert it == ito == 200
    assert np.abs(m - mo).max() < 1e-9
    assert abs(mt - mto) <= 1e-8 * mto
    (it2, mt2), m2 = _run_gpu(deck, m0, method="vpo", timestep=0.1, mass=1.0, conv_torque=1e-6, max_iter=20000,
                              check_every=25)
    mo2 = m0.copy()
    ito2, mto2 = O.minimize_vpo(O.Model(deck), mo2, 0.1, 1.0, 1e-6, 20000)
    assert mt2 < 1e-6 and mto2 < 1e-6
    # over thousands of iterations the momentum of the projection amplifies the
    # rounding of the global sums: the count to convergence differs, and the two
    # stop at different points of the torque < 1e-6 basin (soft in-plane modes),
    # whose energies agree to 1e-7 relative
    assert abs(it2 - ito2) <= 0.15 * ito2
    M = O.Model(deck)
    assert abs(M.energy(m2) - M.energy(mo2)) <= 1e-7 * abs(M.energy(mo2))
    # the reference's norm quirk: the first predictor is not normalised
    assert np.abs(np.linalg.norm(m2, axis=1) - np.linalg.norm(mo2, axis=1)).max() < 1e-12


def test_infinite_damping_sweep_matches_the_oracle_in_colour_order():
    import matjes_b200 as mj

    deck = mj.triangular((36, 30), Bz=1.0)
    m0 = mj.random_sphere(deck.nsites, 23)
    (it, mt, colors), m = _run_gpu(deck, m0, method="infdamp", conv_torque=1e-30, max_iter=60, check_every=20)
    assert it == 60
    assert np.prod(colors) > 1
    mo = m0.copy()
    ito, mto = O.minimize_infdamp(O.Model(deck), mo, 1e-30, 60, colors)
    assert ito == 60
    assert np.abs(m - mo).max() < 1e-10
    assert abs(mt - mto) <= 1e-8 * max(mto, 1e-300)


def test_infinite_damping_reaches_the_reference_minimum():
    """Near a minimum both orders of the sweep converge to the same state."""
    import matjes_b200 as mj

    deck = mj.square_film((40, 32, 1), Jv=1e-3, Dv=0.05e-3, Kv=-0.2e-3, Bz=0.5)
    rng = np.random.default_rng(24)
    m0 = np.tile([0.0, 0.0, 1.0], (deck.nsites, 1)) + 0.2 * rng.standard_normal((deck.nsites, 3))
    m0 /= np.linalg.norm(m0, axis=1, keepdims=True)
    (it, mt, colors), m = _run_gpu(deck, m0, method="infdamp", conv_torque=1e-9, max_iter=20000, check_every=50)
    mo = m0.copy()
    ito, mto = O.minimize_infdamp(O.Model(deck), mo, 1e-9, 20000)  # the reference's site order
    assert mt < 1e-9 and mto < 1e-9
    assert np.abs(m - mo).max() < 1e-6
    M = O.Model(deck)
    assert abs(M.energy(m) - M.energy(mo)) <= 1e-10 * abs(M.energy(mo))


def test_minimisers_reject_what_they_cannot_run():
    import ctypes as C

    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi

    dip = mj.square_film((8, 8, 2), a=0.25, med_z=-0.3, dip=True)
    ham = mj.Hamiltonian(dip)
    m = torch.zeros(3, dip.nsites, dtype=torch.float64, device="cuda")
    p = _abi.MinParams(0.1, 1.0, 1e-6, 10)
    it, mt = C.c_int64(), C.c_double()
    st = _abi.lib.mj_minimize_infdamp(ham.plan, m.data_ptr(), C.byref(p), 5, C.byref(it), C.byref(mt), None, None)
    assert st == _abi.MJ_ERR_UNSUPPORTED
    p0 = _abi.MinParams(0.1, 0.0, 1e-6, 10)
    assert _abi.lib.mj_minimize(ham.plan, m.data_ptr(), C.byref(p0), 5, C.byref(it), C.byref(mt), None) == _abi.MJ_ERR_ARG


def test_run_from_a_reference_input_directory(tmp_path):
    """An input directory in the reference's format (input deck + magnetic_init.dat)
    runs on the GPU and writes EM.dat and magnetic_final.dat; the final state is the
    oracle's SIB trajectory of the same deck."""
    from matjes_b200 import reference_io as R
    from matjes_b200.deck import random_sphere
    from tests.test_reference_io import DECK

    (tmp_path / "input").write_text(DECK)
    ri = R.parse_input(DECK)
    m0 = random_sphere(ri.deck.nsites, 17)
    R.write_order_file(str(tmp_path / "magnetic_init.dat"), m0)
    mT, lines = R.run_dynamics(str(tmp_path))
    assert (tmp_path / "EM.dat").exists() and (tmp_path / "magnetic_final.dat").exists()
    assert len(lines) == 1 + 3   # header + steps 1, 11, 21 (Efreq 10, duration 30)
    m_init = R.read_order_file(str(tmp_path / "magnetic_init.dat"), ri.deck.nsites)
    mo = m_init.copy()
    O.Model(ri.deck).run(mo, 30, integrator="sib", timestep=0.1, alpha=0.3)
    assert np.abs(mT - mo).max() < 1e-9
    back = R.read_order_file(str(tmp_path / "magnetic_final.dat"), ri.deck.nsites)
    assert np.abs(back - mT).max() < 1e-15
