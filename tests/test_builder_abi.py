"""The C ABI library loads and exports its header; the host coupling builder
(the stencil the kernels run) equals the oracle's sparse Hamiltonian (CPU)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from matjes_b200 import _abi
from matjes_b200.deck import Deck, square_areal, square_film, triangular
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "matjes_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mj_[a-z0-9_]+)\s*\(", src)))


def test_every_header_symbol_is_exported_and_bound():
    syms = header_symbols()
    assert len(syms) >= 25
    lib = C.CDLL(_abi.LIB_PATH)
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in include/matjes_gpu.h but not exported"
        assert s in _abi.SIGNATURES, f"{s} has no ctypes signature"
    assert set(_abi.SIGNATURES) <= set(syms)


def test_fortran_binding_names_header_symbols():
    """fortran/matjes_gpu.f90 (the bind(c) module of the Fortran driver; no
    Fortran compiler exists here to build it) binds only names that the header
    declares and the library exports, each with as many dummy arguments as the
    C prototype has parameters."""
    import re

    src = open(os.path.join(ROOT, "fortran", "matjes_gpu.f90")).read()
    hdr = open(os.path.join(ROOT, "include", "matjes_gpu.h")).read()
    syms = header_symbols()
    lib = C.CDLL(_abi.LIB_PATH)
    binds = re.findall(r"function\s+(\w+)\(([^)]*)\)\s*(?:&\s*\n\s*)?bind\(c,\s*name=\"(\w+)\"\)", src)
    assert len(binds) >= 30
    for fname, args, cname in binds:
        if cname == "strlen":
            continue
        assert fname == cname and cname in syms and hasattr(lib, cname), cname
        proto = re.search(r"\b%s\(([^;()]*)\);" % cname, hdr).group(1)
        nparams = 0 if proto.strip() == "void" else proto.count(",") + 1
        nargs = len([a for a in args.split(",") if a.strip()])
        assert nargs == nparams, (cname, nargs, nparams)


def test_version_and_error_strings():
    assert b"sm_100a" in _abi.lib.mj_version()
    assert isinstance(_abi.lib.mj_last_error(), bytes)


def describe(deck):
    lat, h, keep = deck.c_structs()
    n = C.c_int32()
    off = np.zeros(3 * 64, np.int32)
    W = np.zeros(9 * 64)
    W0 = np.zeros(9)
    zc = np.zeros(1)
    st = _abi.lib.mj_stencil_describe(C.byref(lat), C.byref(h), 64, C.byref(n), off.ctypes.data, W.ctypes.data,
                                      W0.ctypes.data, zc.ctypes.data)
    return st, n.value, off[: 3 * n.value].reshape(-1, 3), W[: 9 * n.value].reshape(-1, 3, 3), W0.reshape(3, 3), zc[0]


def oracle_site_tensors(deck, cell):
    """-(H + H^T) blocks of one row site, keyed by column site, from the oracle COO."""
    M = O.Model(deck)
    r, c, v = M.coo()
    out = {}
    for rr, cc, vv in zip(r, c, v):
        if rr // 3 == cell:
            out.setdefault(cc // 3, np.zeros((3, 3)))[rr % 3, cc % 3] -= vv
        if cc // 3 == cell:
            out.setdefault(rr // 3, np.zeros((3, 3)))[cc % 3, rr % 3] -= vv
    return out


def cell_index(deck, x, y, z):
    return x + deck.L[0] * (y + deck.L[1] * z)


DECKS = {
    "square_J_D_K_B": lambda: square_film((12, 12, 1)),
    "triangular_3shells_D1": lambda: triangular((14, 14)),
    "cubic_film_open_z": lambda: square_film((10, 10, 6), a=0.25, med_z=-0.3),
    "tilted_anisotropy": lambda: Deck(L=(9, 7, 1), periodic=(1, 1, 0), areal=square_areal(),
                                      atoms=[((0, 0, 0), 1, 2.0), ((0.5, 0.5, -0.5), 2, 0.0)],
                                      J=[(1, 1, 1, 1e-3), (1, 1, 2, -0.2e-3)], D=[(1, 1, 2, 1, 0.3e-3)],
                                      K=[(1, (1.0, 2.0, 0.5), -0.1e-3)], B_ext=(0.3, -0.2, 0.5)),
}


@pytest.mark.parametrize("name", sorted(DECKS))
def test_stencil_equals_oracle_sparse_hamiltonian(name):
    deck = DECKS[name]()
    st, n, off, W, W0, zc = describe(deck)
    assert st == 0
    # an interior site (all offsets in range along open axes)
    x, y, z = deck.L[0] // 2, deck.L[1] // 2, deck.L[2] // 2
    ref = oracle_site_tensors(deck, cell_index(deck, x, y, z))
    got = {}
    for o, w in zip(off, W):
        j = cell_index(deck, (x + o[0]) % deck.L[0], (y + o[1]) % deck.L[1], (z + o[2]) % deck.L[2])
        got[j] = got.get(j, np.zeros((3, 3))) + w
    i = cell_index(deck, x, y, z)
    got[i] = got.get(i, np.zeros((3, 3))) + W0
    assert set(got) == set(ref)
    scale = max(np.abs(t).max() for t in ref.values())
    for j in ref:
        assert np.abs(got[j] - ref[j]).max() <= 1e-15 * scale, (j, got[j], ref[j])
    assert abs(zc - O.MUB * 2.0) < 1e-20


def test_square_dmi_is_z_cross_bond():
    st, n, off, W, W0, zc = describe(square_film((8, 8, 1), Jv=0.0, Kv=0.0, Bz=0.0))
    for o, w in zip(off, W):
        # antisymmetric part of W encodes B += 2 D (m_j x d): W = 2 D [d]x^T ... d = z x r
        d = np.array([-o[1], o[0], 0.0])
        a = 0.5 * (w - w.T)
        dvec = np.array([a[2, 1], a[0, 2], a[1, 0]])
        assert np.allclose(np.cross(dvec, d), 0, atol=1e-18) and abs(np.dot(dvec, d)) > 1e-5


def test_triangular_shells_and_offsets():
    st, n, off, W, W0, zc = describe(triangular((16, 16)))
    assert n == 18
    nn = {(1, 0), (0, 1), (1, 1), (-1, 0), (0, -1), (-1, -1)}
    second = {(1, -1), (2, 1), (1, 2), (-1, 1), (-2, -1), (-1, -2)}
    third = {(2, 0), (0, 2), (2, 2), (-2, 0), (0, -2), (-2, -2)}
    assert {tuple(o[:2]) for o in off} == nn | second | third
    for o, w in zip(off, W):
        k = tuple(o[:2])
        J = 1e-3 if k in nn else (-0.1e-3 if k in second else -0.05e-3)
        assert abs(np.trace(w) / 3 - 2 * J) < 1e-18
        if k in nn:  # in-plane DMI: no z component of d
            a = 0.5 * (w - w.T)
            assert abs(a[1, 0]) < 1e-20 and abs(a[0, 1]) < 1e-20


def test_multi_atom_cells_are_not_a_stencil():
    deck = Deck(L=(4, 4, 1), periodic=(1, 1, 0), areal=square_areal(),
                atoms=[((0, 0, 0), 1, 2.0), ((0.5, 0.5, 0), 1, 1.0)], J=[(1, 1, 1, 1e-3)])
    st = describe(deck)[0]
    assert st == _abi.MJ_ERR_UNSUPPORTED
    assert b"ELL" in _abi.lib.mj_last_error()


def test_missing_dmi_geometry_is_an_error():
    # an in-plane mediator at the plaquette centre: the two nearest ones cancel on every bond
    deck = Deck(L=(4, 4, 1), periodic=(1, 1, 0), areal=square_areal(), atoms=[((0, 0, 0), 1, 2.0), ((0.5, 0.5, 0), 2, 0.0)],
                J=[(1, 1, 1, 1e-3)], D=[(1, 1, 2, 1, 1e-4)])
    with pytest.raises(RuntimeError):
        O.Model(deck)  # the reference stops: "DID NOT FIND A SINGLE DMI CONTRIBUTION"
    assert describe(deck)[0] == _abi.MJ_ERR_GEOMETRY
