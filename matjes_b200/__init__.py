"""matjes_b200: B200-native (sm_100a, FP64) Matjes spin-dynamics hot path.

The effective field B_eff = -dE/dm (exchange shells, DMI, uniaxial anisotropy,
Zeeman, FFT dipolar) and the LLG time step (Euler, Matjes Heun, SIB; Philox or
injected thermal field) run as hand-written CUDA kernels behind the C ABI of
include/matjes_gpu.h; this package is its host-side mirror of the reference's
Hamiltonian / dynamics interface.  Importing it requires the built
libmatjes_b200.so (``python matjes_b200/build.py``); there is no CPU fallback.
"""
from ._abi import MatjesError, lib  # noqa: F401  (loads the CUDA library or raises)
from .deck import Deck, random_sphere, reversed_disks, square_film, triangular, workload  # noqa: F401
from .hamiltonian import Hamiltonian, SpinDynamics, SpinState, minimize  # noqa: F401
from .batch import ReplicaBatch  # noqa: F401
from .adjoint import SIBTrajectory, deck_terms, field_vjp  # noqa: F401
from .montecarlo import MCInput, MetropolisMC, montecarlo_run, parallel_tempering_run  # noqa: F401

__all__ = ["Deck", "Hamiltonian", "SpinDynamics", "SpinState", "ReplicaBatch", "SIBTrajectory", "minimize", "MatjesError", "workload", "square_film",
           "triangular", "random_sphere", "reversed_disks", "MCInput", "MetropolisMC", "montecarlo_run",
           "parallel_tempering_run"]
