"""Failure bound and step plan of the randomized exclusion certificate (hsolve's verify module,
include/hsolve/verify.hpp:177-188), through the native library. The check itself is
Session.exclusion_check."""
from __future__ import annotations

from . import _native
from . import api as _api  # noqa: F401  (registers the C signatures of include/hsg_solve.h)

__all__ = ["exclusion_failure_bound", "exclusion_block_steps"]


def exclusion_failure_bound(epsilon: float, block_steps: int, dimension: int, block_size: int, kappa: float,
                            complex_scalars: bool = False) -> float:
    """delta(s): bound on P(pass and more than the found eigenvalues within r) after `block_steps` block
    steps of `block_size` columns on a complement of `dimension`, for the relative gap `epsilon`
    (1 for epsilon <= 0, 0 for dimension 0). Raises for block_steps < 1 or kappa < 1."""
    v = _native.lib().hsg_exclusion_failure_bound(float(epsilon), int(block_steps), int(dimension), int(block_size),
                                                  float(kappa), 1 if complex_scalars else 0)
    if v != v:  # NaN: the call failed
        from . import errors

        raise errors.InvalidInputError(_native.lib().hsg_last_error().decode(errors="replace"))
    return v


def exclusion_block_steps(epsilon: float, delta: float, dimension: int, block_size: int, kappa: float,
                          complex_scalars: bool = False) -> int:
    """Smallest s >= 1 whose failure bound is <= delta, at most ceil(dimension / block_size) + 1 (a
    space covering the complement); -1 for epsilon <= 0 or delta outside (0, 1)."""
    return int(_native.lib().hsg_exclusion_block_steps(float(epsilon), float(delta), int(dimension), int(block_size),
                                                       float(kappa), 1 if complex_scalars else 0))
