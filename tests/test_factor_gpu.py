"""GPU parity of the sparse LDL^T through the C ABI (hsolve tests/cpp/test_factor.cpp semantics):
exact Sylvester counts at mid-gap shifts, counts equal to the CPU oracle's and to dense counts,
singular shifts flagged, multi-RHS solves backward stable (<= 1e-12)."""
import numpy as np
import pytest
import scipy.linalg as sla
import scipy.sparse as sp

from hsolve_b200 import Factorization
from hsolve_b200.gen import yee
from oracle import ref, yee_exact
from oracle.ldlt import OracleLDLT
from tests.helpers import laplacian_1d, laplacian_2d, random_spd, random_symmetric, saddle_point

pytestmark = pytest.mark.gpu


def backward_error(k, x, b):
    kn = abs(k).sum(axis=0).max()  # ||K||_1 >= ||K||_2
    r = k @ x - b
    return max(np.linalg.norm(r[:, j]) / (kn * np.linalg.norm(x[:, j])) for j in range(x.shape[1]))


def test_laplacian_1d_exact_inertia():
    n = 600
    a = laplacian_1d(n)
    w = yee_exact.laplacian_1d_spectrum(n)
    f = Factorization()
    f.analyze(a, None, 1.0, -2.0)
    for s in yee_exact.mid_gap_shifts(w, 9, 1e-9):
        assert f.factorize(1.0, -s), s
        inr = f.inertia()
        assert inr.valid and inr.neg == yee_exact.count_below(w, s) and inr.zero == 0 and inr.pos == n - inr.neg


def test_laplacian_2d_exact_inertia_and_solve():
    nx, ny = 60, 45
    a = laplacian_2d(nx, ny)
    n = a.shape[0]
    w = yee_exact.laplacian_2d_spectrum(nx, ny)
    f = Factorization()
    f.analyze(a, None, 1.0, -4.0)
    rng = np.random.default_rng(0)
    for s in yee_exact.mid_gap_shifts(w, 12, 1e-7):
        assert f.factorize(1.0, -s)
        inr = f.inertia()
        assert inr.neg == yee_exact.count_below(w, s) and inr.zero == 0
        b = rng.standard_normal((n, 4))
        x = f.solve(b)
        assert backward_error(a - s * sp.identity(n), x, b) < 1e-12


@pytest.mark.parametrize("cells", [(8, 7, 6), (12, 12, 12)])
def test_yee_exact_inertia_matches_oracle(cells):
    box = yee.Box(cells)
    a, _ = yee.pencil(box)
    n = a.shape[0]
    w = yee_exact.exact_spectrum(cells)
    f = Factorization()
    f.analyze(a, None, 1.0, -25.0)
    o = OracleLDLT(a)
    rng = np.random.default_rng(3)
    shifts = yee_exact.mid_gap_shifts(w[w > 1.0], 8, 1e-6) + [25.0, -3.0]
    for s in shifts:
        assert f.factorize(1.0, -s), s
        inr = f.inertia()
        k = (a - s * sp.identity(n)).tocsr()
        ok, (oneg, ozero, opos), _ = o.factorize(k)
        assert ok
        assert inr.neg == yee_exact.count_below(w, s) == oneg, (s, inr)
        assert inr.zero == ozero == 0
        b = rng.standard_normal((n, 3))
        assert backward_error(k, f.solve(b), b) < 1e-12


def test_generalized_yee_box():
    box = yee.Box((7, 6, 5), (1.0, 0.7, 0.45))
    a, b = yee.pencil(box, "generalized")
    w = yee_exact.exact_spectrum(box.cells, box.lengths)
    f = Factorization()
    f.analyze(a, b, 1.0, -30.0)
    for s in yee_exact.mid_gap_shifts(w[w > 1.0], 6, 1e-6):
        assert f.factorize(1.0, -s)
        assert f.inertia().neg == yee_exact.count_below(w, s)


def test_random_pencils_dense_counts():
    for seed in range(3):
        a = random_symmetric(300, 0.03, seed)
        b = random_spd(300, 0.02, seed + 100)
        w = sla.eigh(a.toarray(), b.toarray(), eigvals_only=True)
        f = Factorization()
        f.analyze(a, b, 1.0, 0.0)
        for s in yee_exact.mid_gap_shifts(w, 8, 1e-6):
            assert f.factorize(1.0, -s)
            assert f.inertia().neg == yee_exact.count_below(w, s), (seed, s)
        # B definiteness test as the driver does it: inertia of 0*A + 1*B
        inr = f.count(0.0, 1.0)
        assert inr.valid and inr.neg == 0 and inr.zero == 0 and inr.pos == 300


def test_saddle_point_needs_pivoting():
    k = saddle_point(400, 150, 5)
    n = k.shape[0]
    w = np.linalg.eigvalsh(k.toarray())
    order = np.empty(n, dtype=np.int32)
    # multipliers first (1-based pivot positions): forces 2x2 pivots / delays
    seq = np.concatenate((np.arange(400, n), np.arange(400)))
    order[seq] = np.arange(1, n + 1)
    f = Factorization()
    f.analyze(k, None, 1.0, 0.0, pivot_order=order)
    assert f.factorize(1.0, 0.0)
    inr = f.inertia()
    assert inr.neg == int((w < 0).sum()) and inr.pos == int((w > 0).sum())
    assert inr.two_by_two + inr.delayed_pivots > 0
    b = np.random.default_rng(2).standard_normal((n, 2))
    assert backward_error(k, f.solve(b), b) < 1e-12


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built (make -C oracle ref)")
def test_factorization_under_the_reference_pivot_order():
    """The GPU factorization analysed with the reference's own nested-dissection PERM_IN (its
    compute_ordering, built from its sources): inertia equal to the exact counts and to the oracle's
    under the same order, and backward-stable solves."""
    box = yee.Box((10, 9, 8))
    a, _ = yee.pencil(box)
    n = a.shape[0]
    w = yee_exact.exact_spectrum(box.cells)
    perm, _ = ref.compute_ordering(a)
    gaps = np.flatnonzero(np.diff(w) > 1e-6 * w[-1])
    shifts = [0.5 * (w[i] + w[i + 1]) for i in (gaps[gaps >= n // 3][0], gaps[gaps >= 2 * n // 3][0])]
    f = Factorization()
    f.analyze(a, None, 1.0, -shifts[0], pivot_order=perm)
    o = OracleLDLT(a, order=np.argsort(perm).astype(np.int32))
    for s in shifts:
        assert f.factorize(1.0, -s)
        inr = f.inertia()
        k = (a - s * sp.identity(n)).tocsr()
        ok, (oneg, ozero, _), _ = o.factorize(k)
        assert ok and inr.valid and inr.neg == oneg == yee_exact.count_below(w, s) and inr.zero == ozero == 0
        b = np.random.default_rng(1).standard_normal((n, 3))
        assert backward_error(k, f.solve(b), b) < 1e-12


def test_singular_shift_flagged(golden):
    z = np.load(golden / "near_singular.npz")
    a = sp.csr_matrix((z["data"], z["indices"], z["indptr"]))
    w = z["eigenvalues"]
    import json
    sigma = json.loads((golden / "examples.json").read_text())["near-singular-shift"]["config"]["target"]["sigma"]
    f = Factorization()
    f.analyze(a, None, 1.0, -sigma)
    assert not f.factorize(1.0, -sigma)
    inr = f.inertia()
    assert not inr.valid and inr.null_pivots >= 1
    with pytest.raises(Exception):
        f.solve(np.ones(a.shape[0]))
    s = yee_exact.mid_gap_shifts(w, 3, 1e-6)[1]
    assert f.factorize(1.0, -s)
    assert f.inertia().neg == yee_exact.count_below(w, s)


def test_count_releases_factors():
    a = laplacian_2d(30, 20)
    f = Factorization()
    f.analyze(a, None, 1.0, -1.0)
    inr = f.count(1.0, -1.0)
    assert inr.valid
    with pytest.raises(Exception):
        f.solve(np.ones(a.shape[0]))
    assert f.factorize(1.0, -1.0)
    f.solve(np.ones(a.shape[0]))


@pytest.mark.parametrize("h", [125, 129, 131, 150, 195])
def test_zero_block_dense_front_two_by_two_solves(h):
    """One dense front K = [[0, B], [B^T, 0]]: its zero blocks stay zero under elimination, so the
    pivots are 2 x 2 pivots and pairs fall across the 128-pivot super-blocks of the large-front
    solve; inertia is exact and solves stay backward stable."""
    rng = np.random.default_rng(h)
    n = 2 * h
    bm = rng.standard_normal((h, h))
    k = sp.bmat([[None, sp.csr_matrix(bm)], [sp.csr_matrix(bm.T), None]]).tocsr()
    f = Factorization()
    f.analyze(k, None, 1.0, 0.0)
    assert f.factorize(1.0, 0.0)
    inr = f.inertia()
    assert inr.two_by_two > n // 4
    evals = np.linalg.eigvalsh(k.toarray())
    assert inr.neg == int((evals < 0).sum())
    b = rng.standard_normal((n, 9))
    x = f.solve(b)
    assert backward_error(k, x, b) < 1e-12


@pytest.mark.parametrize("case", ["yee", "box1e5", "saddle", "singular", "single"])
def test_inertia_only_count_equals_the_factorization(case, golden):
    """hsg_count (fronts factorized level by level in a recycled panel arena, no factor kept) gives
    the inertia of hsg_factorize - exact counts, 2x2 and delayed pivots with re-plans, null pivots
    of a singular shift, FP32 objects - and leaves no usable factorization
    (SparseFactorization::count / InertiaCounter::count, include/hsolve/factor.hpp:383-390)."""
    opts = {}
    if case in ("yee", "single"):
        box = yee.Box((12, 11, 10), (1.0, 0.75, 0.55))
        a, b = yee.pencil(box, "generalized")
        w = yee_exact.exact_spectrum(box.cells, box.lengths)
        shifts = yee_exact.mid_gap_shifts(w[w > 1.0], 5, 1.0)
        order = None
        if case == "single":
            opts = {"precision": 1}
    elif case == "box1e5":
        a, b = yee.pencil(yee.BOX_1E5, "generalized")
        w = yee_exact.exact_spectrum(yee.BOX_1E5.cells, yee.BOX_1E5.lengths)
        shifts, order = [40.0, 120.0, 200.0], None
    elif case == "saddle":
        a, b = saddle_point(400, 150, 5), None
        n = a.shape[0]
        w = np.linalg.eigvalsh(a.toarray())
        order = np.empty(n, dtype=np.int32)
        order[np.concatenate((np.arange(400, n), np.arange(400)))] = np.arange(1, n + 1)
        shifts = [0.0, 0.37]
    else:
        z = np.load(golden / "near_singular.npz")
        a, b = sp.csr_matrix((z["data"], z["indices"], z["indptr"])), None
        import json
        w = z["eigenvalues"]
        shifts = [json.loads((golden / "examples.json").read_text())["near-singular-shift"]["config"]["target"]["sigma"],
                  yee_exact.mid_gap_shifts(w, 3, 1e-6)[1]]
        order = None
    f, c = Factorization(**opts), Factorization(**opts)
    f.analyze(a, b, 1.0, -shifts[0], pivot_order=order)
    c.analyze(a, b, 1.0, -shifts[0], pivot_order=order)
    for s in shifts:
        ok = f.factorize(1.0, -s)
        fi = f.inertia()
        ci = c.count(1.0, -s)
        assert (ci.neg, ci.zero, ci.pos, ci.valid) == (fi.neg, fi.zero, fi.pos, fi.valid), (s, ci, fi)
        assert bool(fi.valid) == bool(ok)
        assert ci.two_by_two == fi.two_by_two
        if case != "saddle" and ok:
            assert ci.neg == yee_exact.count_below(w, s)
        with pytest.raises(Exception):
            c.solve(np.ones(a.shape[0]))
    f.close()
    c.close()
