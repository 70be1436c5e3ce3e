"""CPU: the oracle and the input generator pinned against the reference's own fixtures
(tests/golden, generated by tests/golden/make_golden.py from hsolve's generators and examples)."""
import json

import numpy as np
import pytest
import scipy.linalg as sla
import scipy.sparse as sp

from hsolve_b200.gen import yee
from oracle import yee_exact
from oracle.ldlt import OracleLDLT
from tests.helpers import laplacian_1d, laplacian_2d, random_spd, random_symmetric, saddle_point


def _csr(z, prefix, n):
    return sp.csr_matrix((z[prefix + "_data"], z[prefix + "_indices"], z[prefix + "_indptr"]), shape=(n, n))


def test_exact_spectra_match_reference_formula(golden):
    z = np.load(golden / "yee_spectra.npz")
    names = [k for k in z.files if not k.endswith("__params")]
    assert len(names) >= 6
    for name in names:
        p = z[name + "__params"]
        cells = tuple(int(c) for c in p[:3])
        lengths = tuple(p[3:6])
        phases = tuple(p[6:9])
        boundary = "pec" if p[9] else "bloch"
        w = yee_exact.exact_spectrum(cells, lengths, boundary, phases)
        ref = z[name]
        assert w.shape == ref.shape, name
        np.testing.assert_allclose(w, ref, rtol=1e-13, atol=1e-12 * ref.max(), err_msg=name)


@pytest.mark.parametrize("name,box,form", [
    ("pec_4x3x5", yee.Box((4, 3, 5)), None),
    ("pec_box_5x4x3", yee.Box((5, 4, 3), (1.0, 0.7, 0.45)), None),
    ("bloch_4x3x3", yee.Box((4, 3, 3), (1.0, 0.9, 0.8), "bloch", (0.3 * np.pi, 0.2 * np.pi, 0.1 * np.pi)), None),
])
def test_generator_matches_reference_matrices(golden, name, box, form):
    z = np.load(golden / "yee_matrices.npz")
    n = box.n_edges
    a, b = yee.assemble(box)
    s = yee.standard_form(a, b)
    for tag, mine in (("A", a), ("B", b), ("S", s)):
        ref = _csr(z, f"{name}__{tag}", n)
        assert abs(ref - mine).max() <= 1e-13 * abs(ref).max(), (name, tag)
        assert ((ref != 0) != (mine != 0)).nnz == 0, (name, tag)


def test_generator_matches_reference_inhomogeneous(golden):
    z = np.load(golden / "yee_matrices.npz")
    box = yee.Box((4, 4, 4), (1.0, 1.0, 1.0), "bloch", (0.4 * np.pi, 0.25 * np.pi, 0.1 * np.pi))
    eps = yee.sphere_permittivity(box, 0.25, 12.0)
    np.testing.assert_allclose(eps, z["sphere_4x4x4__eps"], rtol=0, atol=1e-15)
    a, b = yee.assemble(box, eps=eps)
    for tag, mine in (("A", a), ("B", b)):
        ref = _csr(z, f"sphere_4x4x4__{tag}", box.n_edges)
        assert abs(ref - mine).max() <= 1e-13 * abs(ref).max(), tag


def test_generator_rebuilds_reference_examples(golden):
    """The Yee example cases of the reference (examples/cases/*) are rebuilt bit-for-bit in pattern
    and to rounding in values by our generator from their meta.json parameters."""
    ex = json.loads((golden / "examples.json").read_text())
    done = 0
    for name, e in ex.items():
        prm = e["meta"]["params"]
        if prm.get("generator") != "yee" or prm.get("eps", None) != 1.0:
            continue
        box = yee.Box(tuple(prm["cells"]), tuple(prm["lengths"]), prm["boundary"], tuple(prm["phases"]))
        a, b = yee.pencil(box, prm["form"])
        u = sp.csr_matrix(a)
        u.sort_indices()
        dg = e["A_digest"]
        assert u.shape[0] == dg["n"] and u.nnz == dg["nnz"], name
        assert abs(np.abs(u.data).sum() - dg["abs_sum"]) <= 1e-12 * dg["abs_sum"], name
        assert abs(u.diagonal().sum() - dg["trace"]) <= 1e-12 * abs(dg["trace"]), name
        # the reference spectrum near the target is the exact formula's
        w = yee_exact.exact_spectrum(box.cells, box.lengths, box.boundary, box.phases)
        if "ref_nearest" in e:
            sigma = e["config"]["target"]["sigma"]
            order = np.argsort(np.abs(w - sigma), kind="stable")
            mine = np.sort(w[order[: len(e["ref_nearest"])]])
            np.testing.assert_allclose(mine, np.sort(e["ref_nearest"]), rtol=1e-12)
        else:
            lo, hi = e["config"]["target"]["lower"], e["config"]["target"]["upper"]
            inside = w[(w >= lo) & (w <= hi)]
            np.testing.assert_allclose(np.sort(inside), np.sort(e["ref_interval"]), rtol=1e-12)
        done += 1
    assert done >= 4


def test_oracle_inertia_laplacians():
    """hsolve tests/cpp/test_factor.cpp:198-232: exact inertia at mid-gap shifts."""
    n = 600
    a = laplacian_1d(n)
    w = yee_exact.laplacian_1d_spectrum(n)
    o = OracleLDLT(a)
    for s in yee_exact.mid_gap_shifts(w, 9, 1e-9):
        valid, (neg, zero, pos), _ = o.factorize(a - s * sp.identity(n))
        assert valid and neg == yee_exact.count_below(w, s) and zero == 0 and pos == n - neg
    a = laplacian_2d(60, 45)
    w = yee_exact.laplacian_2d_spectrum(60, 45)
    o = OracleLDLT(a)
    for s in yee_exact.mid_gap_shifts(w, 12, 1e-7):
        valid, (neg, zero, pos), _ = o.factorize(a - s * sp.identity(a.shape[0]))
        assert valid and neg == yee_exact.count_below(w, s) and zero == 0


def test_oracle_inertia_yee_and_solve():
    box = yee.Box((8, 7, 6))
    a, _ = yee.pencil(box)
    n = a.shape[0]
    w = yee_exact.exact_spectrum(box.cells)
    o = OracleLDLT(a)
    shifts = yee_exact.mid_gap_shifts(w[w > 1.0], 6, 1e-6) + [25.0, -3.0]
    for s in shifts:
        k = (a - s * sp.identity(n)).tocsr()
        valid, (neg, zero, pos), st = o.factorize(k)
        assert valid and neg == yee_exact.count_below(w, s), s
        b = np.random.default_rng(1).standard_normal((n, 3))
        x = o.solve(b)
        kn = abs(k).sum(axis=0).max()
        be = np.abs(k @ x - b).max() / (kn * np.abs(x).max())
        assert be < 1e-13, (s, be)


def test_oracle_dense_counts_random_and_saddle():
    for seed in range(3):
        a = random_symmetric(250, 0.03, seed)
        w = np.linalg.eigvalsh(a.toarray())
        o = OracleLDLT(a)
        for s in yee_exact.mid_gap_shifts(w, 6, 1e-6):
            valid, (neg, _, _), _ = o.factorize(a - s * sp.identity(250))
            assert valid and neg == yee_exact.count_below(w, s)
    k = saddle_point(150, 60, 3)
    w = np.linalg.eigvalsh(k.toarray())
    # zero-diagonal multipliers eliminated first: needs 2x2 pivots and delays
    order = np.concatenate((np.arange(150, 210), np.arange(150))).astype(np.int32)
    o = OracleLDLT(k, order=order)
    valid, (neg, zero, pos), st = o.factorize(k)
    assert valid and neg == int((w < 0).sum()) and pos == int((w > 0).sum())
    assert st["two_by_two"] + st["delayed"] > 0


def test_oracle_generalized_pencil():
    a = random_symmetric(200, 0.04, 11)
    b = random_spd(200, 0.03, 12)
    w = sla.eigh(a.toarray(), b.toarray(), eigvals_only=True)
    o = OracleLDLT(a + b)
    for s in yee_exact.mid_gap_shifts(w, 8, 1e-6):
        valid, (neg, _, _), _ = o.factorize(a - s * b)
        assert valid and neg == yee_exact.count_below(w, s)


def test_oracle_near_singular_shift_is_flagged(golden):
    """examples near-singular-shift: sigma 1e-12 (relative) from an eigenvalue -> singular K."""
    z = np.load(golden / "near_singular.npz")
    a = sp.csr_matrix((z["data"], z["indices"], z["indptr"]))
    w = z["eigenvalues"]
    ex = __import__("json").loads((golden / "examples.json").read_text())["near-singular-shift"]
    sigma = ex["config"]["target"]["sigma"]
    o = OracleLDLT(a)
    valid, _, st = o.factorize(a - sigma * sp.identity(a.shape[0]))
    assert not valid and st["null_pivots"] >= 1
    # a shift in a spectral gap is exact
    s = yee_exact.mid_gap_shifts(w, 3, 1e-6)[1]
    valid, (neg, _, _), _ = o.factorize(a - s * sp.identity(a.shape[0]))
    assert valid and neg == yee_exact.count_below(w, s)


def test_complex_embedding_recovers_hermitian_eigenpairs():
    """The real 2n embedding of a complex Hermitian pencil and the recovery of its eigenpairs
    (clusters of doubled eigenvalues -> B-orthonormal complex vectors) against numpy's complex
    eigensolver, on the CPU with the embedded problem solved densely."""
    from hsolve_b200.api import _embed, _unembed

    rng = np.random.default_rng(5)
    n = 40
    m = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    a = sp.csr_matrix(m + m.conj().T)
    r = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = sp.csr_matrix(r @ r.conj().T + n * np.eye(n))
    ae, be = _embed(a).toarray(), _embed(b).toarray()
    assert np.allclose(ae, ae.T) and np.allclose(be, be.T)
    w, v = sla.eigh(ae, be)
    lam_ref = sla.eigh(a.toarray(), b.toarray(), eigvals_only=True)
    np.testing.assert_allclose(w[0::2], lam_ref, rtol=1e-10, atol=1e-10)  # every eigenvalue twice
    np.testing.assert_allclose(w[1::2], lam_ref, rtol=1e-10, atol=1e-10)
    sel = slice(10, 20)  # ten embedded pairs = five complex eigenpairs
    report = {"scale": 1.0, "norm2_a": float(np.linalg.norm(a.toarray(), 2)),
              "norm2_b": float(np.linalg.norm(b.toarray(), 2)),
              "certificate": {"count_inertia": 10, "count_found": 10, "passed": True}}
    lam, x, rep = _unembed(w[sel], v[:, sel], report, a, b, 1e-10, "interval", 0.0, 0)
    np.testing.assert_allclose(lam, lam_ref[5:10], rtol=1e-10)
    np.testing.assert_allclose(x.conj().T @ (b @ x), np.eye(5), atol=1e-10)
    assert rep["success"] and rep["certificate"]["count_inertia"] == 5
    assert all(p["backward_error"] < 1e-12 for p in rep["pairs"])
