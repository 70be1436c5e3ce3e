"""hsolve_b200 - B200-native shift-invert eigensolver path of hsolve (sparse LDL^T with inertia,
multi-RHS solves, block orthogonalisation, residual SpMV) behind hsolve's API."""
from __future__ import annotations

from . import errors
from ._native import Factorization, Inertia, compute_ordering, symbolic_stats
from .errors import *  # noqa: F401,F403

__all__ = ["Factorization", "Inertia", "compute_ordering", "symbolic_stats", *[c.__name__ for c in errors.ERROR_CLASSES],
           "HsolveError", "HsolveWarning"]
