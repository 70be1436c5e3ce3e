"""GPU: the mixed-precision path - FP32 operator factorizations with FP64 iterative refinement of every
shift-invert application, FP64 inertia counts (hsolve's factor_precision = single,
include/hsolve/solver.hpp:116-126; the refinement of src/ops/shift_invert_operator.cpp:83-177; the
reference's own check that a refined single factor reaches double accuracy,
tests/cpp/test_ops.cpp:164-330).

* An FP32 factorization through the C ABI (precision = 1) has the inertia of the oracle at mid-gap
  shifts, and its unrefined solve is accurate to FP32 rounding (backward error up to ~1e-4, not 1e-13).
* hsolve_b200.solve(..., factor_precision="single") on Yee and Nedelec pencils: every refined
  application converges, the eigenvalues equal the exact spectrum (Yee) or the FP64 path's (Nedelec)
  within 1e-10 relative, every pair's backward error is <= 1e-10, the certificate counts are the
  FP64 ones, and the report says single precision was used.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import hsolve_b200 as hsolve
from hsolve_b200 import _native
from hsolve_b200.gen import nedelec, yee
from oracle import yee_exact
from oracle.ldlt import OracleLDLT

pytestmark = pytest.mark.gpu

EIG_RTOL = 1e-10


def _backward_error(k, x, b):
    return np.abs(k @ x - b).max() / (abs(k).sum(axis=0).max() * np.abs(x).max() + np.abs(b).max())


@pytest.mark.parametrize("cells,form", [((9, 8, 7), "standard"), ((14, 11, 8), "generalized")])
def test_fp32_factorization_inertia_and_unrefined_accuracy(cells, form):
    box = yee.Box(cells, (1.0, 0.75, 0.55))
    a, b = yee.pencil(box, form)
    bb = b if form == "generalized" else sp.identity(a.shape[0], format="csr")
    w = yee_exact.exact_spectrum(box.cells, box.lengths)
    shifts = yee_exact.mid_gap_shifts(w[w > 1.0], 4, 1.0)  # gaps far above FP32 rounding of K
    f32 = _native.Factorization(device=0, precision=1)
    f32.analyze(a, b if form == "generalized" else None, 1.0, -shifts[0])
    o = OracleLDLT(a + bb)
    for s in shifts:
        k = (a - s * bb).tocsr()
        ok, (neg, zero, _), _ = o.factorize(k)
        assert ok and zero == 0
        assert f32.factorize(1.0, -s)
        inr = f32.inertia()
        assert inr.valid and inr.neg == neg == yee_exact.count_below(w, s), (s, inr, neg)
        rhs = np.random.default_rng(1).standard_normal((a.shape[0], 3))
        x = f32.solve(rhs)
        be = _backward_error(k, x, rhs)
        assert 1e-12 < be < 1e-3, be  # FP32 rounding (about 1e3 eps32, as FP64 factors reach 1e3 eps64)
    f32.close()


def _check(res, tol=1e-10):
    assert res.success, res.report
    for pr in res.report["pairs"]:
        assert pr["backward_error"] <= tol, pr


def test_single_precision_interval_matches_exact_spectrum():
    box = yee.Box((14, 11, 8), (1.0, 0.75, 0.55))
    a, b = yee.pencil(box, "generalized")
    w = yee_exact.exact_spectrum(box.cells, box.lengths)
    # a low-frequency window: eps32 * cond(K) well below 1, so the refinement contracts (deep in the
    # dense upper spectrum it need not, and the solve falls back to FP64 factors; tested below)
    cuts = yee_exact.mid_gap_shifts(w[(w > 1.0) & (w < 300.0)], 10, 1e-6)
    lo, hi = cuts[2], cuts[5]
    res = hsolve.solve(a, b, lower=lo, upper=hi, config={"factor_precision": "single"})
    _check(res)
    prec = res.report["precision"]
    assert prec["requested"] == "single" and prec["used"] == "single" and not prec["fallback"], prec
    assert prec["refinement"]["applies"] > 0 and prec["refinement"]["steps"] > 0
    want = w[(w >= lo) & (w <= hi)]
    np.testing.assert_allclose(res.eigenvalues, want, rtol=EIG_RTOL)
    cert = res.report["certificate"]
    assert cert["passed"] and cert["count_inertia"] == want.size
    x = res.eigenvectors
    assert np.abs(x.T @ (b @ x) - np.eye(want.size)).max() < 1e-10


def test_single_precision_nearest_matches_exact_spectrum():
    box = yee.Box((12, 12, 12))
    a, _ = yee.pencil(box)
    w = yee_exact.exact_spectrum(box.cells)
    sigma = 47.3
    res = hsolve.solve(a, sigma=sigma, k=8, config={"factor_precision": "single"})
    _check(res)
    assert res.report["precision"]["used"] == "single"
    order = np.argsort(np.abs(w - sigma), kind="stable")
    np.testing.assert_allclose(np.sort(res.eigenvalues), np.sort(w[order[:8]]), rtol=EIG_RTOL)
    assert res.report["certificate"]["passed"]


def test_single_precision_nedelec_matches_double_path():
    a, b = nedelec.pencil(nedelec.TetBox((24, 12, 6)))
    lo, hi = 40.0, 90.0
    r64 = hsolve.solve(a, b, lower=lo, upper=hi)
    r32 = hsolve.solve(a, b, lower=lo, upper=hi, config={"factor_precision": "single"})
    _check(r64)
    _check(r32)
    assert r32.report["precision"]["used"] == "single"
    assert r32.eigenvalues.size == r64.eigenvalues.size > 0
    np.testing.assert_allclose(r32.eigenvalues, r64.eigenvalues, rtol=EIG_RTOL)
    assert r32.report["certificate"]["count_inertia"] == r64.report["certificate"]["count_inertia"]


def test_single_precision_falls_back_to_double_where_refinement_cannot_converge():
    """Deep in the dense upper spectrum eps32 * cond(K) approaches 1: the refinement of an
    application stops without converging, the FP32 attempt is abandoned and the solve reruns with
    FP64 factors (hsolve's rule, include/hsolve/solver.hpp:116-126): the result is still certified
    and exact, and the report says why single precision was not used."""
    box = yee.Box((14, 11, 8), (1.0, 0.75, 0.55))
    a, b = yee.pencil(box, "generalized")
    w = yee_exact.exact_spectrum(box.cells, box.lengths)
    cuts = yee_exact.mid_gap_shifts(w[w > 1.0], 10, 1e-6)
    lo, hi = cuts[2], cuts[5]
    res = hsolve.solve(a, b, lower=lo, upper=hi, config={"factor_precision": "single"})
    _check(res)
    prec = res.report["precision"]
    assert prec["requested"] == "single"
    if prec["used"] == "double":
        assert "did not converge" in prec["fallback"] or "not accepted" in prec["fallback"]
    np.testing.assert_allclose(res.eigenvalues, w[(w >= lo) & (w <= hi)], rtol=EIG_RTOL)
