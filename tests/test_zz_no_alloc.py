"""mj_energy_noalloc: the total energy with no device allocation.

Some callers cannot call cudaMalloc when they evaluate the energy, for
instance a host code whose GPU memory is handed out by its own pool or capped
by its job scheduler once it is set up.  This entry point keeps its reduction
scratch in a fixed static device array instead of the plan's buffers.  The
tests call it through the C ABI twice in a row (the array keeps the previous
call's partial sums, so the second call must not see them) and compare with
mj_energy, the existing entry point, at the energy tolerance of the other GPU
tests (1e-12 relative).  This file is collected last on purpose.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _noalloc(ham, m_t):
    import torch

    from matjes_b200 import _abi

    E = torch.full((1,), float("nan"), dtype=torch.float64, device=m_t.device)
    _abi.check(_abi.lib.mj_energy_noalloc(ham.plan, m_t.data_ptr(), E.data_ptr(),
                                          torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return float(E.item())


def _decks():
    import matjes_b200 as mj

    two_atom = mj.Deck(L=(24, 20, 1), periodic=(1, 1, 0), areal=np.eye(3),
                       atoms=[((0, 0, 0), 1, 2.0), ((0.5, 0.5, 0), 1, 1.5), ((0.5, 0.0, -0.5), 2, 0.0)],
                       J=[(1, 1, 1, 1e-3), (1, 1, 2, 0.4e-3)], D=[(1, 1, 2, 1, 0.2e-3)], K=[(1, (0, 0, 1), -0.1e-3)],
                       B_ext=(0, 0, 0.7))
    return {"triangular_1024": mj.triangular((1024, 1024)), "square_odd": mj.square_film((97, 61, 1)),
            "two_atom_cell": two_atom}


@pytest.mark.parametrize("name", ["triangular_1024", "square_odd", "two_atom_cell"])
def test_noalloc_energy_matches_mj_energy_on_two_calls(name):
    import torch

    import matjes_b200 as mj

    deck = _decks()[name]
    ham = mj.Hamiltonian(deck)
    m1 = mj.random_sphere(deck.nsites, 1)
    m2 = mj.random_sphere(deck.nsites, 2)
    E1_ref = ham.energy(m1)  # the existing entry point (mj_energy)
    E2_ref = ham.energy(m2)
    t1 = torch.tensor(m1.T.copy(), device="cuda")
    t2 = torch.tensor(m2.T.copy(), device="cuda")
    a = _noalloc(ham, t1)
    b = _noalloc(ham, t1)  # second call in a row, same input
    c = _noalloc(ham, t2)  # and on a different state
    assert abs(a - E1_ref) <= TOL * abs(E1_ref)
    assert abs(b - E1_ref) <= TOL * abs(E1_ref)
    assert a == b
    assert abs(c - E2_ref) <= TOL * abs(E2_ref)


def test_noalloc_rejects_what_it_cannot_hold():
    import torch

    import matjes_b200 as mj
    from matjes_b200 import _abi

    big = mj.square_film((4096, 4104, 1))  # 128 x 513 blocks of 32 x 8 sites > MJ_NOALLOC_MAX_BLOCKS
    ham = mj.Hamiltonian(big)
    m = torch.zeros(3, big.nsites, dtype=torch.float64, device="cuda")
    E = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = _abi.lib.mj_energy_noalloc(ham.plan, m.data_ptr(), E.data_ptr(), None)
    assert st == _abi.MJ_ERR_ARG and b"MJ_NOALLOC_MAX_BLOCKS" in _abi.lib.mj_last_error()
    del ham
    dip = mj.square_film((8, 8, 4), a=0.25, med_z=-0.3, dip=True)
    hd = mj.Hamiltonian(dip)
    md = torch.zeros(3, dip.nsites, dtype=torch.float64, device="cuda")
    assert _abi.lib.mj_energy_noalloc(hd.plan, md.data_ptr(), E.data_ptr(), None) == _abi.MJ_ERR_UNSUPPORTED
