"""Per-site field and energy of the CUDA kernels against the oracle (1e-12 relative)."""
import numpy as np
import pytest

from conftest import scalar_rel_err, site_rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _decks():
    from matjes_b200.deck import Deck, square_areal, square_film, triangular

    return {
        "square64_cfg": lambda: square_film((64, 64, 1)),
        "triangular64_3shells": lambda: triangular((64, 64)),
        "film16x16x6_open_z": lambda: square_film((16, 16, 6), Jv=1e-3, Dv=0.15e-3, Kv=-0.02e-3, Bz=0.2, a=0.25,
                                                  med_z=-0.3),
        "odd_5x7": lambda: square_film((5, 7, 1)),
        "tiny_triangular_3x3": lambda: triangular((3, 3)),
        "chain_open": lambda: square_film((17, 1, 1), Dv=0.0, periodic=(0, 0, 0)),
        "open_square_9x6": lambda: square_film((9, 6, 1), periodic=(0, 0, 0)),
        "tilted_axis_inplane_B": lambda: Deck(L=(12, 10, 1), periodic=(1, 1, 0), areal=square_areal(),
                                              atoms=[((0, 0, 0), 1, 2.0), ((0.5, 0.5, -0.5), 2, 0.0)],
                                              J=[(1, 1, 1, 1e-3), (1, 1, 2, -0.2e-3)], D=[(1, 1, 2, 1, 0.3e-3)],
                                              K=[(1, (1.0, 2.0, 0.5), -0.1e-3)], B_ext=(0.3, -0.2, 0.5)),
        "two_atom_cell_ell": lambda: Deck(L=(6, 5, 1), periodic=(1, 1, 0), areal=square_areal(),
                                          atoms=[((0, 0, 0), 1, 2.0), ((0.5, 0.5, 0), 1, 1.5), ((0.5, 0.0, -0.5), 2, 0.0)],
                                          J=[(1, 1, 1, 1e-3), (1, 1, 2, 0.4e-3)], D=[(1, 1, 2, 1, 0.2e-3)],
                                          K=[(1, (0, 0, 1), -0.1e-3)], B_ext=(0, 0, 0.7)),
    }


DECK_NAMES = ["square64_cfg", "triangular64_3shells", "film16x16x6_open_z", "odd_5x7", "tiny_triangular_3x3",
              "chain_open", "open_square_9x6", "tilted_axis_inplane_B", "two_atom_cell_ell"]


def variants(ham):
    """Kernel variants of a plan: -1 generic, 0..5 tiled (when a shape matched)."""
    from matjes_b200 import _abi

    v, s = _abi.C.c_int32(), _abi.C.c_int32()
    _abi.check(_abi.lib.mj_plan_get_variant(ham.plan, _abi.C.byref(v), _abi.C.byref(s)))
    return [-1, 0, 1, 2, 3, 4, 5] if s.value else [-1]


def set_variant(ham, v):
    from matjes_b200 import _abi

    _abi.check(_abi.lib.mj_plan_set_variant(ham.plan, v))


@pytest.mark.parametrize("name", DECK_NAMES)
def test_field_energy_match_oracle(name):
    import matjes_b200 as mj

    deck = _decks()[name]()
    ham = mj.Hamiltonian(deck)
    M = O.Model(deck)
    m = mj.random_sphere(deck.nsites, 11)
    Bo, eo = M.field(m)
    Eo = M.energy(m)
    from matjes_b200 import _abi

    for v in variants(ham):
        for tma in ((0, 1) if v >= 0 else (0,)):
            if ham.noffsets:
                set_variant(ham, v)
                _abi.check(_abi.lib.mj_plan_set_tma(ham.plan, tma))
            B, e = ham.get_eff_field(m, with_energy=True)
            assert site_rel_err(B, Bo) < TOL, (v, tma)
            assert scalar_rel_err(e, eo) < TOL, (v, tma)
            assert abs(ham.energy(m) - Eo) <= TOL * abs(Eo), (v, tma)
            _abi.check(_abi.lib.mj_plan_check_status(ham.plan))


def test_shapes_are_matched():
    import matjes_b200 as mj
    from matjes_b200 import _abi

    def shape(deck):
        v, s = _abi.C.c_int32(), _abi.C.c_int32()
        _abi.check(_abi.lib.mj_plan_get_variant(mj.Hamiltonian(deck).plan, _abi.C.byref(v), _abi.C.byref(s)))
        return s.value

    assert shape(mj.square_film((16, 16, 1))) == 1
    assert shape(mj.triangular((16, 16), J=(1e-3,))) == 2
    assert shape(mj.triangular((16, 16))) == 3
    sq2 = mj.square_film((16, 16, 1))
    sq2.J.append((1, 1, 2, -0.1e-3))
    assert shape(sq2) == 4
    assert shape(mj.square_film((8, 8, 4), med_z=-0.3)) == 0  # z couplings: generic kernel


@pytest.mark.parametrize("variant", [-1, 0, 1, 2, 3])
def test_square_nnn_variants(variant):
    import matjes_b200 as mj

    deck = mj.square_film((40, 24, 1))
    deck.J.append((1, 1, 2, -0.1e-3))
    ham = mj.Hamiltonian(deck)
    set_variant(ham, variant)
    m = mj.random_sphere(deck.nsites, 12)
    Bo, eo = O.Model(deck).field(m)
    B, e = ham.get_eff_field(m, with_energy=True)
    assert site_rel_err(B, Bo) < TOL and scalar_rel_err(e, eo) < TOL


def test_per_site_bfield_map():
    import matjes_b200 as mj

    deck = mj.square_film((32, 32, 1))
    rng = np.random.default_rng(3)
    b = np.zeros((deck.ncell, 3))
    b[:, 2] = 0.5 + rng.normal(0, 0.05, deck.ncell)
    b[:, 0] = 0.1 * np.sin(np.arange(deck.ncell))
    ham = mj.Hamiltonian(deck)
    ham.set_bfield(b)
    M = O.Model(deck)
    M.set_bfield(b)
    m = mj.random_sphere(deck.nsites, 2)
    B, e = ham.get_eff_field(m, with_energy=True)
    Bo, eo = M.field(m)
    assert site_rel_err(B, Bo) < TOL and scalar_rel_err(e, eo) < TOL


def test_coo_plan_from_reference_triplets():
    """The cuda_H_init route: the oracle's 1-based COO handed to mj_plan_from_coo."""
    import matjes_b200 as mj

    deck = mj.triangular((10, 12))
    M = O.Model(deck)
    r, c, v = M.coo()
    zee = np.full(deck.nsites, -O.MUB * 2.0)
    bsite = np.tile(deck.B_ext, (deck.nsites, 1))
    ham = mj.Hamiltonian.from_coo(deck.nsites, r + 1, c + 1, v, base=1, zeeman=zee, b_site=bsite)
    m = mj.random_sphere(deck.nsites, 4)
    B, e = ham.get_eff_field(m, with_energy=True)
    Bo, eo = M.field(m)
    assert site_rel_err(B, Bo) < TOL and scalar_rel_err(e, eo) < TOL


def test_device_tensor_interface_matches_host():
    import torch

    import matjes_b200 as mj

    deck = mj.triangular((48, 40))
    ham = mj.Hamiltonian(deck)
    m = mj.random_sphere(deck.nsites, 9)
    Bh = ham.get_eff_field(m)
    mt = torch.tensor(m.T.copy(), device="cuda")
    Bt = ham.get_eff_field(mt)
    torch.cuda.synchronize()
    assert np.array_equal(Bt.cpu().numpy().T, Bh)


def test_full_size_uniform_and_translation_properties():
    """cfg size 1024^2 triangular: a ferromagnet gives the analytic field on every
    site; a shifted state gives the shifted field (translation invariance)."""
    import torch

    import matjes_b200 as mj

    deck = mj.triangular((1024, 1024))
    ham = mj.Hamiltonian(deck)
    N = deck.nsites
    m = torch.zeros(3, N, dtype=torch.float64, device="cuda")
    m[2] = 1.0
    B, e = ham.get_eff_field(m, with_energy=True)
    bz = 2 * (6 * 1e-3 + 6 * -0.1e-3 + 6 * -0.05e-3) + 2 * 0.05e-3 + O.MUB * 2.0
    assert torch.allclose(B[2], torch.full_like(B[2], bz), rtol=1e-14, atol=0)
    assert B[:2].abs().max().item() < 1e-18
    e_exp = -(6 * 1e-3 + 6 * -0.1e-3 + 6 * -0.05e-3) + (-0.05e-3) - O.MUB * 2.0
    assert abs(e.sum().item() - N * e_exp) < 1e-12 * N * abs(e_exp)
    g = torch.Generator(device="cuda").manual_seed(0)
    r = torch.randn(3, N, dtype=torch.float64, device="cuda", generator=g)
    r = r / r.norm(dim=0, keepdim=True)
    B1 = ham.get_eff_field(r)
    shift = lambda t: torch.roll(t.view(3, 1024, 1024), shifts=(37, 11), dims=(1, 2)).reshape(3, N)  # noqa: E731
    B2 = ham.get_eff_field(shift(r).contiguous())
    assert torch.equal(B2, shift(B1))


def test_full_size_sampled_sites_against_oracle_tensors():
    """1024^2 triangular random state: 2000 sampled sites against the oracle's
    per-site tensors (translation-invariant couplings taken from a 16^2 build)."""
    import torch

    import matjes_b200 as mj

    from test_builder_abi import oracle_site_tensors

    L = 1024
    deck = mj.triangular((L, L))
    small = mj.triangular((16, 16))
    ref = oracle_site_tensors(small, 8 + 16 * 8)
    offs = []
    for j, T in ref.items():
        ox, oy = j % 16 - 8, j // 16 - 8
        offs.append((ox, oy, T))
    ham = mj.Hamiltonian(deck)
    m = mj.random_sphere(deck.nsites, 21)
    B = ham.get_eff_field(torch.tensor(m.T.copy(), device="cuda")).cpu().numpy().T
    rng = np.random.default_rng(1)
    mm = m.reshape(L, L, 3)
    for _ in range(2000):
        x, y = rng.integers(0, L, 2)
        b = np.zeros(3)
        for ox, oy, T in offs:
            b += T @ mm[(y + oy) % L, (x + ox) % L]
        b += O.MUB * 2.0 * np.array(deck.B_ext)
        got = B[x + L * y]
        assert np.linalg.norm(got - b) <= TOL * max(np.linalg.norm(b), 1e-3 * 0.01)
