"""Failure reports of the device status word, made to happen without a GPU fault.

* A bounded device wait that gives up: mj_plan_selftest_timeout arms an
  mbarrier for bytes that no copy delivers (nothing is issued, so nothing is in
  flight) and polls it a few times through the same bounded wait as the tiled
  kernels' TMA staging.  mj_plan_check_status must then report MJ_ERR_TIMEOUT
  once, clear the word, and leave the plan usable (energies and steps equal to
  those of a plan that never saw the timeout).
* A non-finite spin: a NaN planted in the host state must come back as
  MJ_ERR_NAN from mj_plan_check_status after an asynchronous step (tiled and
  generic kernels, every integrator) and from mj_step_host itself (the striped
  one-step path from pinned memory and the plain path).
* mj_gneb_path reads the word after its relaxation and returns the report.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plan(L=32):
    import matjes_b200 as mj

    deck = mj.triangular((L, L))
    return deck, mj.Hamiltonian(deck)


def test_bounded_wait_gives_up_reports_timeout_and_the_plan_stays_usable():
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi

    deck, ham = _plan()
    m0 = mj.random_sphere(deck.nsites, 5)
    E0 = ham.energy(m0)
    assert _abi.lib.mj_plan_check_status(ham.plan) == _abi.MJ_OK
    _abi.check(_abi.lib.mj_plan_selftest_timeout(ham.plan, 64, None))
    assert _abi.lib.mj_plan_check_status(ham.plan) == _abi.MJ_ERR_TIMEOUT
    assert b"bounded device wait" in _abi.lib.mj_last_error()
    # reported once: the word is cleared
    assert _abi.lib.mj_plan_check_status(ham.plan) == _abi.MJ_OK
    assert ham.energy(m0) == E0
    # steps after the report equal those of a fresh plan
    ref = mj.Hamiltonian(deck)
    a = torch.tensor(m0.T.copy(), device="cuda")
    b = a.clone()
    mj.SpinDynamics(ham, integrator="sib", timestep=0.1, alpha=0.1).run(a, 5)
    mj.SpinDynamics(ref, integrator="sib", timestep=0.1, alpha=0.1).run(b, 5)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    # the argument range is checked
    assert _abi.lib.mj_plan_selftest_timeout(ham.plan, 0, None) == _abi.MJ_ERR_ARG


@pytest.mark.parametrize("integrator", ["sib", "heun", "euler"])
@pytest.mark.parametrize("variant", [-1, 4])
def test_nonfinite_spin_is_reported_after_an_asynchronous_step(integrator, variant):
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi

    deck, ham = _plan()
    _abi.check(_abi.lib.mj_plan_set_variant(ham.plan, variant))
    m0 = mj.random_sphere(deck.nsites, 6)
    sd = mj.SpinDynamics(ham, integrator=integrator, timestep=0.1, alpha=0.1)
    good = torch.tensor(m0.T.copy(), device="cuda")
    sd.run(good, 2)
    assert _abi.lib.mj_plan_check_status(ham.plan) == _abi.MJ_OK
    m0[100, 1] = np.nan
    bad = torch.tensor(m0.T.copy(), device="cuda")
    sd.run(bad, 1)
    assert _abi.lib.mj_plan_check_status(ham.plan) == _abi.MJ_ERR_NAN
    assert b"non-finite" in _abi.lib.mj_last_error()
    assert _abi.lib.mj_plan_check_status(ham.plan) == _abi.MJ_OK


@pytest.mark.parametrize("pinned", [True, False])
def test_host_step_returns_the_nonfinite_report(pinned):
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi

    deck, ham = _plan()
    sd = mj.SpinDynamics(ham, integrator="sib", timestep=0.1, alpha=0.1)
    m0 = mj.random_sphere(deck.nsites, 7)
    host = torch.tensor(m0, dtype=torch.float64)
    if pinned:
        host = host.pin_memory()
    E = np.empty(1)
    _abi.check(_abi.lib.mj_step_host(ham.plan, host.data_ptr(), _abi.C.byref(sd.p), 1, E.ctypes.data))
    host[3, 2] = float("inf")
    st = _abi.lib.mj_step_host(ham.plan, host.data_ptr(), _abi.C.byref(sd.p), 1, E.ctypes.data)
    assert st == _abi.MJ_ERR_NAN
    assert _abi.lib.mj_plan_check_status(ham.plan) == _abi.MJ_OK
    host.copy_(torch.tensor(m0))
    _abi.check(_abi.lib.mj_step_host(ham.plan, host.data_ptr(), _abi.C.byref(sd.p), 1, E.ctypes.data))


def test_gneb_path_returns_a_pending_timeout():
    import matjes_b200 as mj
    from matjes_b200 import _abi
    from matjes_b200.gneb import PlanPath, geodesic_path

    deck = mj.square_film((8, 8, 1), Jv=1e-3, Dv=0.4e-3, Kv=-0.2e-3, Bz=0.3)
    n = deck.nsites
    up = np.tile([0.0, 0.0, 1.0], (n, 1))
    path = geodesic_path(up, -up, 6, amp_rnd=1e-2, seed=1)
    path[0], path[-1] = up, -up
    holder = PlanPath(mj.Hamiltonian(deck), path)
    _abi.check(_abi.lib.mj_plan_selftest_timeout(holder.ham.plan, 16, None))
    with pytest.raises(mj.MatjesError):
        holder.gneb_path(0.3, 0.02, 1.0, 0.0, 10, "I")
    assert b"bounded device wait" in _abi.lib.mj_last_error()
    # the report cleared the word: the next relaxation runs
    holder.gneb_path(0.3, 0.02, 1.0, 0.0, 10, "I")
