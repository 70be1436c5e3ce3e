"""CPU: the CPU port of the whole certified solve (oracle/cpu_path.py), which the bench times as the
reference's CPU path, reproduces exact Yee spectra with its certificates; the faster oracle
(relaxed supernodes, blocked fronts, parallel tree) keeps exact inertia and FP64 solves."""
import numpy as np
import scipy.sparse as sp

from hsolve_b200.gen import yee
from oracle import cpu_path, yee_exact
from oracle.ldlt import OracleLDLT


def test_relaxed_oracle_inertia_and_solve_match_the_fundamental_one():
    box = yee.Box((12, 10, 9), (1.0, 0.75, 0.55))
    a, b = yee.pencil(box, "generalized")
    w = yee_exact.exact_spectrum(box.cells, box.lengths)
    pattern = (abs(a) + abs(b)).tocsr()
    o0, o1 = OracleLDLT(pattern), OracleLDLT(pattern, relax=True)
    assert o1.supernodes < o0.supernodes
    rhs = np.random.default_rng(2).standard_normal((a.shape[0], 5))
    for s in yee_exact.mid_gap_shifts(w[w > 1.0], 5, 1e-3):
        k = (a - s * b).tocsr()
        (ok0, in0, _), (ok1, in1, _) = o0.factorize(k), o1.factorize(k)
        assert ok0 and ok1 and in0 == in1 and in0[0] == yee_exact.count_below(w, s)
        x0, x1 = o0.solve(rhs), o1.solve(rhs)
        assert np.abs(x0 - x1).max() <= 1e-9 * np.abs(x0).max()
        be = np.abs(k @ x1 - rhs).max() / (abs(k).sum(axis=0).max() * np.abs(x1).max())
        assert be < 1e-12


def test_cpu_path_interval_and_nearest_match_exact_spectra():
    box = yee.Box((12, 10, 9), (1.0, 0.75, 0.55))
    a, b = yee.pencil(box, "generalized")
    w = yee_exact.exact_spectrum(box.cells, box.lengths)
    cuts = yee_exact.mid_gap_shifts(w[w > 1.0], 10, 1e-6)
    P = cpu_path.CpuPencil(a, b)
    lam, x, rep = cpu_path.solve_interval(P, cuts[2], cuts[5])
    want = w[(w >= cuts[2]) & (w <= cuts[5])]
    assert rep["success"] and rep["count_inertia"] == want.size == lam.size
    np.testing.assert_allclose(lam, want, rtol=1e-10)
    assert np.abs(x.T @ (b @ x) - np.eye(want.size)).max() < 1e-10
    lam, _, rep = cpu_path.solve_nearest(P, 61.7, 6)
    order = np.argsort(np.abs(w - 61.7), kind="stable")
    assert rep["success"]
    np.testing.assert_allclose(np.sort(lam), np.sort(w[order[:6]]), rtol=1e-10)


def test_cpu_path_standard_form_identity_b():
    a, _ = yee.pencil(yee.Box((8, 7, 6)))
    w = yee_exact.exact_spectrum((8, 7, 6))
    rep = cpu_path.certified_solve(a, None, {"sigma": 30.0, "k": 4})
    assert rep["success"] and rep["count_found"] == rep["count_inertia"]
    assert sp.issparse(a) and rep["factorizations"] >= 3
    assert np.isfinite(w).all()
