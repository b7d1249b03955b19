"""The triangular ten-shell Hamiltonian with hollow-site DMI, pinned to the
reference's own minimisation run.

Fixture: tests/golden/minimization_triangular100.{json,npz}, made by
make_golden_minimization.py from tests/serial/minimization/{inp, lattice.in,
SpinSTMi.dat, REF} of the Matjes tree (a 100 x 100 triangular monolayer, ten
exchange shells J_1..J_10, nearest-neighbour DMI through the hollow-site atom
at (2/3, 1/3, -0.76), easy axis 0.7 meV, 20 T, mu_s = 3).  Two numbers of that
log pin the Hamiltonian:

* the energy of the start state, printed to 6 decimals (-0.067544 eV/cell):
  the shell counts (6 or 12 neighbours per shell), the J signs, the anisotropy
  and the Zeeman term (mu_s = 3) each move it well past its last digit, and so
  does the sign of D (D = -1 meV gives -0.067527);
* the converged energy of the minimiser, -0.06755225425 eV/cell at a torque of
  1e-5 (the last iterates still fall by 2.5e-11 each, 1 % less per iterate, so
  the minimum lies about 1.2e-9 eV/cell below it).  The start state relaxes into
  a skyrmion whose energy depends on D at first order: a 5 % change of D moves
  it by 9e-7 eV/cell and D = -1 meV unwinds it (-0.0675572, the ferromagnet).
  The reference's log comes from an older minimiser than solvers/minimize.F90,
  so its iterates are not compared: only where they end.
"""
import json
import os

import numpy as np
import pytest

from matjes_b200.deck import Deck
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def fixture():
    with open(os.path.join(HERE, "golden", "minimization_triangular100.json")) as f:
        g = json.load(f)
    k = np.load(os.path.join(HERE, "golden", "minimization_triangular100.npz"))["spins"]
    return g, k.astype(np.float64) / 1e8


def deck_of(g, D_scale=1.0) -> Deck:
    d = g["deck"]
    return Deck(L=tuple(d["L"]), periodic=tuple(d["periodic"]), areal=np.asarray(d["areal"]),
                atoms=[(tuple(a[0]), a[1], a[2]) for a in d["atoms"]], J=[tuple(j) for j in d["J"]],
                D=[(t1, t2, tm, s, v * D_scale) for t1, t2, tm, s, v in d["D"]],
                K=[(t, tuple(ax), v) for t, ax, v in d["K"]], B_ext=tuple(d["B_ext"]), zeeman_on=True)


def converged_energy(model, m, ncell):
    m = m.copy()
    O.minimize_vpo(model, m, 1.0, 1.0, 1e-7, 4000)
    return model.energy(m) / ncell, m


def test_start_energy_matches_the_logged_digits():
    g, m = fixture()
    ncell = 100 * 100
    E = O.Model(deck_of(g)).energy(m) / ncell
    assert abs(E - g["start_energy_per_cell"]) <= 0.5e-6, E
    # the printed digits resolve the DMI sign
    E_flip = O.Model(deck_of(g, -1.0)).energy(m) / ncell
    assert abs(E_flip - g["start_energy_per_cell"]) > 1e-5, E_flip


def test_converged_energy_matches_the_log():
    g, m = fixture()
    ncell = 100 * 100
    E_log = g["iterate_energy_per_cell"][-1]
    E, m_min = converged_energy(O.Model(deck_of(g)), m, ncell)
    # below the log's still-falling last iterate, by about the remaining descent
    assert -3e-9 <= E - E_log <= 0.0, (E, E_log)
    # a skyrmion: spins turned fully in-plane somewhere
    assert np.linalg.norm(m_min[:, :2], axis=1).max() > 0.99
    # the converged energy resolves D to well under a percent
    E5, _ = converged_energy(O.Model(deck_of(g, 1.05)), m, ncell)
    assert abs(E5 - E_log) > 5e-7, E5


# ----------------------------------------------------------------------
# the same pins through the product (C ABI, device kernels)
@pytest.mark.gpu
def test_device_field_and_energy_equal_the_oracle_on_the_pinned_deck():
    import torch

    import matjes_b200 as mj
    from conftest import scalar_rel_err, site_rel_err

    g, m = fixture()
    deck = deck_of(g)
    ham = mj.Hamiltonian(deck)
    mt = torch.tensor(m.T.copy(), device="cuda")
    B, e = ham.get_eff_field(mt, with_energy=True)
    Bo, eo = O.Model(deck).field(m)
    assert site_rel_err(B.cpu().numpy().T, Bo) < 1e-12
    assert scalar_rel_err(e.cpu().numpy(), eo) < 1e-12
    E = ham.energy(mt) / 1e4
    assert abs(E - g["start_energy_per_cell"]) <= 0.5e-6


@pytest.mark.gpu
def test_device_minimiser_ends_at_the_logged_energy():
    import torch

    import matjes_b200 as mj

    g, m = fixture()
    deck = deck_of(g)
    ham = mj.Hamiltonian(deck)
    mt = torch.tensor(m.T.copy(), device="cuda")
    it, tq = mj.minimize(ham, mt, method="vpo", timestep=1.0, mass=1.0, conv_torque=1e-7, max_iter=4000,
                         check_every=50)
    E = ham.energy(mt) / 1e4
    E_log = g["iterate_energy_per_cell"][-1]
    assert -3e-9 <= E - E_log <= 0.0, (E, E_log, it, tq)
