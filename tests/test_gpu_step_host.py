"""One step from and to host memory (mj_step_host) with the copies, transposes
and passes cut into stripes of tile rows.

With pinned host memory the step runs striped; it must equal the unstriped
device step bit for bit (spins and energy): the same per-site arithmetic, the
same block ids and energy partials summed in the same order.  Pageable memory
takes the unstriped path; multi-step calls too."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch

    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    t.numpy()[...] = a
    return t


def _device_step(ham, m0, kw, energy_mode, step0):
    """The unstriped reference: mj_step_dev on the device copy, plain staging."""
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi

    sd = mj.SpinDynamics(ham, **kw)
    sd.p.energy_mode = energy_mode
    sd.p.step0 = step0
    m = torch.tensor(m0.T.copy(), device="cuda")
    E = torch.empty(1, dtype=torch.float64, device="cuda")
    _abi.check(_abi.lib.mj_step_dev(ham.plan, m.data_ptr(), _abi.C.byref(sd.p), 1, E.data_ptr(), None))
    torch.cuda.synchronize()
    return m.cpu().numpy().T.copy(), float(E.item())


CASES = {
    # 1000 rows: the last stripe and the last tile row are partial
    "tri3_sib_thermal": (lambda mj: mj.triangular((96, 1000)), dict(integrator="sib", temperature=10.0, noise="philox",
                                                                     alpha=0.1, timestep=0.1, seed=5)),
    "square_heun_thermal": (lambda mj: mj.square_film((64, 200, 1)), dict(integrator="heun", temperature=20.0,
                                                                          noise="philox", alpha=0.3, seed=2)),
    "square_euler": (lambda mj: mj.square_film((64, 136, 1)), dict(integrator="euler", alpha=0.2)),
    "square_open_y_sib": (lambda mj: mj.square_film((48, 160, 1), periodic=(1, 0, 0)),
                          dict(integrator="sib", temperature=5.0, noise="philox", alpha=0.5, seed=9)),
    "tri_nn_sib": (lambda mj: mj.triangular((64, 256), J=(1e-3,)), dict(integrator="sib", alpha=0.1)),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("energy_mode", [0, 1])
def test_striped_host_step_equals_the_device_step(name, energy_mode):
    import matjes_b200 as mj
    from matjes_b200 import _abi

    make, kw = CASES[name]
    deck = make(mj)
    ham = mj.Hamiltonian(deck)
    _abi.check(_abi.lib.mj_plan_set_tma(ham.plan, 0))
    m0 = mj.random_sphere(deck.nsites, 3)
    want_m, want_E = _device_step(ham, m0, kw, energy_mode, 41)
    for variant in (4, 0, 5):
        _abi.check(_abi.lib.mj_plan_set_variant(ham.plan, variant))
        want_m, want_E = _device_step(ham, m0, kw, energy_mode, 41)
        host = _pinned(m0)
        sd = mj.SpinDynamics(ham, **kw)
        sd.p.energy_mode = energy_mode
        E = sd.run(host.numpy(), 1, energies=True, step0=41)
        assert np.array_equal(host.numpy(), want_m), (name, variant)
        assert E[0] == want_E, (name, variant, E[0], want_E)
        # pageable memory: the unstriped path, the same result
        page = m0.copy()
        sd2 = mj.SpinDynamics(ham, **kw)
        sd2.p.energy_mode = energy_mode
        E2 = sd2.run(page, 1, energies=True, step0=41)
        assert np.array_equal(page, want_m) and E2[0] == want_E


def test_striped_host_steps_chain_and_skip_energy():
    """Consecutive one-step calls continue the trajectory of a multi-step device
    run; no energy requested is allowed."""
    import torch

    import matjes_b200 as mj

    deck = mj.triangular((128, 128))
    ham = mj.Hamiltonian(deck)
    m0 = mj.random_sphere(deck.nsites, 8)
    kw = dict(integrator="sib", temperature=15.0, noise="philox", alpha=0.2, seed=4)
    host = _pinned(m0)
    sd = mj.SpinDynamics(ham, **kw)
    for _ in range(5):
        sd.run(host.numpy(), 1)
    dev = torch.tensor(m0.T.copy(), device="cuda")
    mj.SpinDynamics(ham, **kw).run(dev, 5)
    np.testing.assert_allclose(host.numpy(), dev.cpu().numpy().T, rtol=0, atol=1e-15)


def test_replayed_host_step_follows_buffer_and_parameter_changes():
    """The striped step is captured once per host buffer, coefficients and kernel
    configuration and replayed: alternating two pinned buffers and two
    temperatures, each call equals the device step of the same input, step
    index and parameters."""
    import matjes_b200 as mj

    deck = mj.triangular((96, 200))
    ham = mj.Hamiltonian(deck)
    bufs = [_pinned(mj.random_sphere(deck.nsites, s)) for s in (11, 12)]
    for call in range(6):
        kw = dict(integrator="sib", temperature=(5.0, 30.0)[call % 2], noise="philox", alpha=0.1, seed=7)
        host = bufs[(call // 2) % 2]
        m_in = host.numpy().copy()
        want_m, want_E = _device_step(ham, m_in, kw, 0, 100 + call)
        sd = mj.SpinDynamics(ham, **kw)
        sd.p.energy_mode = 0
        E = sd.run(host.numpy(), 1, energies=True, step0=100 + call)
        assert np.array_equal(host.numpy(), want_m), call
        assert E[0] == want_E, call


@pytest.mark.parametrize("stripes,zerocopy", [(2, 1), (3, 1), (5, 1), (9, 1), (64, 1), (3, 0), (9, 0)])
def test_any_stripe_count_equals_the_device_step(stripes, zerocopy):
    """Every stripe count (64 is clamped to 5 tile rows per stripe) gives the
    device step bit for bit: SIB at 10 K with the energy after the step (three
    chained passes, the first shifted by two tile rows) and before it; the
    stepped spins written by kernels into the mapped host buffer (zerocopy 1)
    or transposed on the device and copied (0)."""
    import matjes_b200 as mj
    from matjes_b200 import _abi

    deck = mj.triangular((96, 1000))
    ham = mj.Hamiltonian(deck)
    _abi.check(_abi.lib.mj_plan_set_option(ham.plan, _abi.MJ_OPT_HOST_STRIPES, stripes))
    _abi.check(_abi.lib.mj_plan_set_option(ham.plan, _abi.MJ_OPT_HOST_ZEROCOPY, zerocopy))
    kw = dict(integrator="sib", temperature=10.0, noise="philox", alpha=0.1, timestep=0.1, seed=5)
    m0 = mj.random_sphere(deck.nsites, 21)
    for energy_mode in (1, 0):
        want_m, want_E = _device_step(ham, m0, kw, energy_mode, 7)
        host = _pinned(m0)
        sd = mj.SpinDynamics(ham, **kw)
        sd.p.energy_mode = energy_mode
        E = sd.run(host.numpy(), 1, energies=True, step0=7)
        assert np.array_equal(host.numpy(), want_m), (stripes, energy_mode)
        assert E[0] == want_E, (stripes, energy_mode)
