"""CPU: this project's ordering, symbolic analysis and residual formula against the reference's own
code for those parts (built from its sources into oracle/_ref by `make -C oracle ref`; skipped where
it was not built): its nested dissection (include/hsolve/factor.hpp:631) and its shifted residual /
SpMM (include/hsolve/sparse.hpp:140-174).
"""
import numpy as np
import pytest
import scipy.sparse as sp

from hsolve_b200 import _native
from hsolve_b200.gen import yee
from oracle import ref, yee_exact
from oracle.ldlt import OracleLDLT

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built (make -C oracle ref)")


def test_reference_order_is_a_pivot_order_our_analysis_accepts():
    a, b = yee.pencil(yee.Box((9, 8, 7), (1.0, 0.8, 0.7)), "generalized")
    perm, top = ref.compute_ordering(a, b)
    n = a.shape[0]
    assert np.array_equal(np.sort(perm), np.arange(1, n + 1)) and 0 < top < n
    st = _native.symbolic_stats(a + b, perm, amalgamate=False)
    o = OracleLDLT(a + b, order=np.argsort(perm).astype(np.int32))
    o.factorize(a + b)                                  # SPD: no delays
    assert st["nnz_l"] == o.nnz_l
    assert abs(st["flops"] - o.flops) <= 1e-9 * o.flops


@pytest.mark.parametrize("box, form, bound", [
    (yee.BOX_1E4, "generalized", 1.05),
    (yee.Box((14, 14, 14)), "standard", 1.20),
])
def test_our_ordering_against_the_reference(box, form, bound):
    """Fill of this project's nested dissection within `bound` of the reference's on the same pencil
    (measured: 1.000 on BOX_1E4, 1.02 on the 1e5 box, 1.12 on the 20^3 cube)."""
    a, b = yee.pencil(box, form)
    pat = a if b is None else a + b
    perm, _ = ref.compute_ordering(a, b)
    theirs = _native.symbolic_stats(pat, perm)["flops"]
    ours = _native.symbolic_stats(pat, None)["flops"]
    assert ours <= bound * theirs, ours / theirs


def test_inertia_does_not_depend_on_whose_order():
    box = yee.Box((8, 7, 6))
    a, _ = yee.pencil(box)
    w = yee_exact.exact_spectrum(box.cells)
    n = a.shape[0]
    perm, _ = ref.compute_ordering(a)
    gaps = np.flatnonzero(np.diff(w) > 1e-6 * w[-1])          # midpoints of distinct neighbours
    for i in (gaps[gaps >= 40][0], gaps[gaps >= 200][0]):
        sigma = 0.5 * (w[i] + w[i + 1])
        k = (a - sigma * sp.identity(n)).tocsr()
        ok1, in1, _ = OracleLDLT(a, order=np.argsort(perm).astype(np.int32)).factorize(k)
        ok2, in2, _ = OracleLDLT(a).factorize(k)
        assert ok1 and ok2 and in1 == in2 and in1[0] == yee_exact.count_below(w, sigma)


@pytest.mark.parametrize("generalized", [False, True])
def test_shifted_residual_formula(generalized):
    a, b = yee.pencil(yee.Box((7, 6, 5)), "generalized" if generalized else "standard")
    n = a.shape[0]
    rng = np.random.default_rng(3)
    x = rng.standard_normal((n, 5))
    y = rng.standard_normal((n, 5))
    sigma = 12.5
    r, omega = ref.shifted_residual(a, b if generalized else None, sigma, x, y)
    bm = b if generalized else sp.identity(n, format="csr")
    expect = bm @ x - (a @ y - sigma * (bm @ y))
    scale = np.abs(bm) @ np.abs(x + sigma * y) + np.abs(a) @ np.abs(y)
    np.testing.assert_allclose(r, expect, rtol=0, atol=1e-13 * np.abs(scale).max())
    np.testing.assert_allclose(omega, (np.abs(r) / scale).max(axis=0), rtol=1e-12)


def test_spmm():
    a, _ = yee.pencil(yee.Box((6, 6, 6)))
    x = np.random.default_rng(4).standard_normal((a.shape[0], 3))
    np.testing.assert_allclose(ref.spmm(a, x), a @ x, rtol=1e-14, atol=1e-12)
