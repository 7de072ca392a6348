"""pinq_b200 — Python binding of libinqb200, the sm_100a implementation of INQ's
Kohn-Sham Hamiltonian application and real-time propagators.

It reaches the same C ABI as the C++ host adapter (``host/inq_b200.hpp``).
"""
from ._lib import FP64, MIXED, THEORY_HARTREE, THEORY_LDA, THEORY_NONE, InqbError, lib  # noqa: F401
from .hamiltonian import KSHamiltonian, build_gaussian_kb, gaussian_beta, grid_supported, sphere  # noqa: F401
from . import systems  # noqa: F401
from .batch import CellBatch  # noqa: F401
from .propagate import propagate  # noqa: F401

__all__ = ["KSHamiltonian", "CellBatch", "propagate", "build_gaussian_kb", "gaussian_beta", "grid_supported", "sphere", "systems",
           "FP64", "MIXED", "THEORY_NONE", "THEORY_HARTREE", "THEORY_LDA", "InqbError", "lib"]
