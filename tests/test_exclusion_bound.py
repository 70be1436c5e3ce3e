"""Failure bound and step plan of the randomized exclusion certificate (hsolve's verify module,
include/hsolve/verify.hpp:177-188) through the C ABI, on CPU: the bound against an independent
evaluation of its formula, minimal and monotone step plans, the step counts the reference's header
quotes and its tests pin (tests/cpp/test_certfast.cpp:50-121), and the edge cases."""
import math

import pytest

from hsolve_b200 import errors
from hsolve_b200.verify import exclusion_block_steps, exclusion_failure_bound


def _formula(eps, s, big_n, p, kappa, cplx):
    """The bound written out in plain double arithmetic (parameters where nothing overflows)."""
    x1 = (2.0 + eps) / (2.0 - eps)
    t1 = math.cosh((s - 1) * math.acosh(x1))
    t = (2.0 - eps) / (eps * t1 * t1 + 2.0 - eps)
    if s >= 2:
        q = (1.0 - eps) ** 2
        e2 = 1.0 - q
        t2 = math.cosh(((s - 2) // 2) * math.acosh((1.0 + e2) / (1.0 - e2)))
        t = min(t, q / (e2 * t2 * t2 + q))
    f = (big_n - 1) * kappa * t if cplx else math.sqrt(big_n * kappa * t)
    return min(f, 1.0) ** p


@pytest.mark.parametrize("cplx", [False, True])
def test_bound_matches_the_formula(cplx):
    for eps in (0.05, 0.3, 0.7):
        for s in (1, 2, 3, 6, 11):
            for p in (1, 3):
                got = exclusion_failure_bound(eps, s, 5000, p, 4.0, cplx)
                want = _formula(eps, s, 5000, p, 4.0, cplx)
                assert got == pytest.approx(want, rel=1e-12, abs=1e-300), (eps, s, p)


@pytest.mark.parametrize("cplx", [False, True])
def test_steps_reach_delta_and_are_minimal(cplx):
    big_n = 100000
    for eps in (0.02, 0.25, 0.6, 0.99):
        for p in (1, 4):
            for delta in (1e-6, 1e-12):
                s = exclusion_block_steps(eps, delta, big_n, p, 1.0, cplx)
                assert s >= 1
                assert exclusion_failure_bound(eps, s, big_n, p, 1.0, cplx) <= delta
                if s > 1:
                    assert exclusion_failure_bound(eps, s - 1, big_n, p, 1.0, cplx) > delta
                for t in range(1, s + 5):  # more steps never hurt
                    assert exclusion_failure_bound(eps, t, big_n, p, 1.0, cplx) >= \
                        exclusion_failure_bound(eps, t + 1, big_n, p, 1.0, cplx)


def test_header_example_step_counts():
    # real, N = 1e5, kappa = 1, p = 1 (include/hsolve/verify.hpp:72-73)
    assert exclusion_block_steps(0.99, 1e-12, 100000, 1, 1.0) == 8
    assert exclusion_block_steps(0.25, 1e-6, 100000, 1, 1.0) == 28
    assert exclusion_block_steps(0.25, 1e-12, 100000, 1, 1.0) == 46


def test_steps_grow_the_expected_way():
    def steps(eps, n, p, kappa, cplx):
        return exclusion_block_steps(eps, 1e-10, n, p, kappa, cplx)
    assert steps(0.1, 100000, 1, 1.0, False) > steps(0.5, 100000, 1, 1.0, False)     # gap
    assert steps(0.3, 1000000, 1, 1.0, False) >= steps(0.3, 1000, 1, 1.0, False)     # log N
    assert steps(0.3, 100000, 1, 1e4, False) >= steps(0.3, 100000, 1, 1.0, False)    # log kappa
    assert steps(0.3, 100000, 1, 1.0, True) <= steps(0.3, 100000, 1, 1.0, False)     # complex
    assert steps(0.3, 100000, 4, 1.0, False) < steps(0.3, 100000, 1, 1.0, False)     # blocks


def test_edge_cases():
    assert exclusion_failure_bound(0.0, 10, 1000, 1, 1.0) == 1.0
    assert exclusion_block_steps(-0.1, 1e-6, 1000, 1, 1.0) == -1
    assert exclusion_block_steps(0.5, 1.5, 1000, 1, 1.0) == -1
    assert exclusion_block_steps(1e-9, 1e-12, 40, 4, 1.0) == 11  # a plan covering the complement
    assert exclusion_failure_bound(0.5, 3, 0, 1, 1.0) == 0.0
    with pytest.raises(errors.InvalidInputError):
        exclusion_failure_bound(0.5, 0, 10, 1, 1.0)
    with pytest.raises(errors.InvalidInputError):
        exclusion_failure_bound(0.5, 1, 10, 1, 0.5)
