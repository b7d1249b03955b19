"""A plain torch float64 restatement of the SIB trajectory, for autograd checks.

Test infrastructure only.  The field is B = -sum_t v_t (H_t + H_t^T) m + zc b,
with H_t the oracle's coupling matrix (COO, AoS mode index 3 i + c) of a deck
holding term t alone at value 1; the SIB stage is the closed-form Cayley solve
of Mentink et al. (2010), y = m + 2/(1+|h|^2) (m x h + (m x h) x h).
"""
from __future__ import annotations

import dataclasses

import numpy as np
import torch

from oracle import oracle as O

HBAR = 0.658211928
MUB = 0.0000578838180661
KB = 0.000086173324


def unit_matrices(deck):
    """Dense (H_t + H_t^T) of every J, D, K term of `deck` at value 1 (AoS 3N x 3N)."""
    n3 = 3 * deck.nsites
    out = []
    terms = [("J", i) for i in range(len(deck.J))] + [("D", i) for i in range(len(deck.D))] + \
            [("K", i) for i in range(len(deck.K))]
    for kind, i in terms:
        J = [deck.J[i][:-1] + (1.0,)] if kind == "J" else []
        D = [deck.D[i][:-1] + (1.0,)] if kind == "D" else []
        K = [deck.K[i][:-1] + (1.0,)] if kind == "K" else []
        d = dataclasses.replace(deck, J=J, D=D, K=K, B_ext=(0.0, 0.0, 0.0), zeeman_on=False)
        r, c, v = O.Model(d).coo()
        H = np.zeros((n3, n3))
        np.add.at(H, (r, c), v)
        out.append(torch.tensor(H + H.T, dtype=torch.float64))
    return out


def zeeman_coefficient(deck) -> float:
    mu = [a[2] for a in deck.atoms if a[2] > 0][0]
    return -(1.0 * MUB * deck.c_zeeman) * mu


def sib_solve(m, p, H, alpha, hc):
    np2 = (p * p).sum(-1, keepdim=True)
    pn = torch.where(np2 > 1e-16, p / torch.sqrt(np2), p)
    h = hc * (H + alpha * torch.cross(pn, H, dim=-1))
    u = torch.cross(m, h, dim=-1)
    c = 2.0 / (1.0 + (h * h).sum(-1, keepdim=True))
    return m + c * (u + torch.cross(u, h, dim=-1))


def trajectory(m0, terms, b, A, zc, nsteps, timestep, alpha, noise=None):
    """m0, b: (N, 3); terms: (nterm,); noise: list of (N, 3) thermal fields per step or None."""
    hc = -0.5 * (timestep / HBAR) / (1.0 + alpha * alpha)

    def field(m):
        mv = m.reshape(-1)
        Bmm = -sum(t * (At @ mv) for t, At in zip(terms, A))
        return Bmm.reshape(-1, 3) + zc * b

    m = m0
    for k in range(nsteps):
        bt = noise[k] if noise is not None else 0.0
        H1 = field(m) + bt
        mb = 0.5 * (m + sib_solve(m, m, H1, alpha, hc))
        H2 = field(mb) + bt
        m = sib_solve(m, mb, H2, alpha, hc)
    return m
