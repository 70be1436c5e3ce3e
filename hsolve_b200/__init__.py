"""hsolve_b200 - B200-native shift-invert eigensolver path of hsolve (sparse LDL^T with inertia,
multi-RHS solves, block orthogonalisation, residual SpMV) behind hsolve's API:

    import hsolve_b200 as hsolve
    res = hsolve.solve(A, B, sigma=25.0, k=10)          # nearest k, exact inertia certificate
    res = hsolve.solve(A, B, lower=40.0, upper=200.0)   # all eigenvalues in an interval
"""
from __future__ import annotations

from . import errors
from ._native import Factorization, Inertia, compute_ordering, symbolic_stats
from .api import Session, SolveResult, solve
from .errors import (FactorizationFailedError, HsolveError, HsolveIOError, HsolveWarning, InternalError,
                     InvalidInputError, NotConvergedError, NotHermitianError, OutOfMemoryBudgetError, SingularError,
                     UnsupportedError)

__all__ = ["solve", "Session", "SolveResult", "Factorization", "Inertia", "compute_ordering", "symbolic_stats", "errors",
           "HsolveError", "InvalidInputError", "HsolveIOError", "NotHermitianError", "UnsupportedError",
           "FactorizationFailedError", "SingularError", "OutOfMemoryBudgetError", "NotConvergedError",
           "InternalError", "HsolveWarning"]
