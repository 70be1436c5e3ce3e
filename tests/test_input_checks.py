"""Input normalization and the Hermitian check of the public API (host code, no GPU).

The fast forms in hsolve_b200.api work on the CSR arrays; these tests hold them to the plain scipy
formulation of the same contract (hsolve's `storage` modes, the relative Frobenius defect
||M - M^H||_F / ||M||_F against hermitian_tol, and the symmetrized (M + M^H) / 2 returned when the
defect is positive but below the tolerance).
"""
import numpy as np
import pytest
import scipy.sparse as sp

from hsolve_b200 import api
from hsolve_b200.errors import NotHermitianError


def _plain_as_csr(m, storage):
    m = sp.csr_matrix(m, copy=True)
    if np.iscomplexobj(m.data):
        m = sp.csr_matrix(m, dtype=np.complex128)
        if not np.any(m.data.imag != 0):
            m = sp.csr_matrix(m.real)
    else:
        m = sp.csr_matrix(m, dtype=np.float64)
    m.sum_duplicates()
    m.eliminate_zeros()
    if storage == "upper":
        m = sp.triu(m) + sp.triu(m, 1).conj().T
    elif storage == "lower":
        m = sp.tril(m) + sp.tril(m, -1).conj().T
    elif storage == "auto":
        up, lo = sp.triu(m, 1).nnz, sp.tril(m, -1).nnz
        if (up == 0) != (lo == 0):
            m = sp.triu(m) + sp.triu(m, 1).conj().T if lo == 0 else sp.tril(m) + sp.tril(m, -1).conj().T
    m = sp.csr_matrix(m)
    m.sum_duplicates()
    m.sort_indices()
    return m


def _plain_defect(m):
    d = m - m.conj().T
    nrm = np.sqrt((np.abs(m.data) ** 2).sum())
    return np.sqrt((np.abs(d.data) ** 2).sum()) / nrm if nrm > 0 else 0.0


def _sym(n, density, seed, complex_=False):
    rng = np.random.default_rng(seed)
    r = sp.random(n, n, density=density, random_state=rng, format="csr")
    if complex_:
        r = r + 1j * sp.random(n, n, density=density, random_state=rng, format="csr")
    return (r + r.conj().T + sp.identity(n)).tocsr()


def _same(x, y):
    assert x.shape == y.shape
    np.testing.assert_array_equal(x.toarray(), y.toarray())


@pytest.mark.parametrize("storage", ["auto", "full", "upper", "lower"])
def test_symmetric_input_all_storages(storage):
    m = _sym(120, 0.05, 1)
    if storage == "upper":
        m_in = sp.triu(m).tocsr()
    elif storage == "lower":
        m_in = sp.tril(m).tocsr()
    else:
        m_in = m
    got = api._as_csr(m_in, "A", storage)
    _same(got, _plain_as_csr(m_in, storage))
    assert got.has_sorted_indices and got.has_canonical_format
    h, defect = api._hermitian_check(got, "A", 1e-10)
    assert defect == 0.0 and h is got
    np.testing.assert_array_equal(h.toarray(), m.toarray())


@pytest.mark.parametrize("half", ["upper", "lower"])
def test_auto_completes_one_triangle(half):
    m = _sym(90, 0.08, 2)
    tri = (sp.triu(m) if half == "upper" else sp.tril(m)).tocsr()
    got = api._as_csr(tri, "A", "auto")
    np.testing.assert_array_equal(got.toarray(), m.toarray())


def test_zeros_duplicates_and_no_mutation():
    rng = np.random.default_rng(3)
    n = 60
    i = rng.integers(0, n, 400)
    j = rng.integers(0, n, 400)
    v = rng.standard_normal(400)
    v[::7] = 0.0                                   # explicit zeros
    coo = sp.coo_matrix((np.r_[v, v], (np.r_[i, j], np.r_[j, i])), shape=(n, n))  # duplicates on the diagonal
    csr = coo.tocsr()                              # tocsr sums duplicates; build an un-summed one too
    raw = sp.csr_matrix((np.r_[v, v, 0.0], (np.r_[i, j, 0], np.r_[j, i, 1])), shape=(n, n))
    for m in (coo, csr, raw):
        before = (m.copy().toarray(), getattr(m, "nnz", None))
        got = api._as_csr(m, "A", "auto")
        _same(got, _plain_as_csr(m, "auto"))
        assert not np.any(got.data == 0)
        after = (m.toarray(), getattr(m, "nnz", None))
        np.testing.assert_array_equal(before[0], after[0])
        assert before[1] == after[1]               # the caller's matrix keeps its stored entries


def test_dense_and_complex_inputs():
    m = _sym(40, 0.2, 4)
    _same(api._as_csr(m.toarray(), "A", "auto"), _plain_as_csr(m, "auto"))
    h = _sym(50, 0.1, 5, complex_=True)
    got = api._as_csr(h, "A", "auto")
    assert np.iscomplexobj(got.data)
    _same(got, _plain_as_csr(h, "auto"))
    hh, defect = api._hermitian_check(got, "A", 1e-10)
    assert defect == 0.0
    real_as_complex = sp.csr_matrix(m, dtype=np.complex128)
    assert not np.iscomplexobj(api._as_csr(real_as_complex, "A", "auto").data)


@pytest.mark.parametrize("complex_", [False, True])
def test_near_hermitian_is_symmetrized(complex_):
    m = _sym(80, 0.06, 6, complex_)
    rng = np.random.default_rng(7)
    noise = m.copy()
    noise.data = noise.data * (1e-13 * rng.standard_normal(noise.nnz))   # same pattern, unsymmetric values
    p = api._as_csr(m + noise, "A", "full")
    expect = _plain_defect(p)
    got, defect = api._hermitian_check(p, "A", 1e-10)
    assert defect > 0 and abs(defect - expect) <= 1e-12 * expect
    np.testing.assert_allclose(got.toarray(), 0.5 * (p + p.conj().T).toarray(), rtol=0, atol=1e-15)
    assert _plain_defect(got) == 0.0


def test_unsymmetric_pattern():
    m = _sym(70, 0.07, 8).tolil()
    m[0, 5] = m[0, 5] + 1e-14 if m[0, 5] != 0 else 1e-14
    m[5, 0] = 0.0
    p = api._as_csr(m.tocsr(), "A", "full")
    expect = _plain_defect(p)
    got, defect = api._hermitian_check(p, "A", 1e-10)
    assert abs(defect - expect) <= 1e-12 * max(expect, 1e-300)
    assert _plain_defect(got) == 0.0


def test_not_hermitian_raises():
    m = _sym(30, 0.1, 9).tolil()
    m[2, 7] = m[2, 7] + 1.0
    with pytest.raises(NotHermitianError):
        api._hermitian_check(api._as_csr(m.tocsr(), "A", "full"), "A", 1e-10)


@pytest.mark.parametrize("case", ["symmetric", "near", "upper_only", "zeros", "unsorted", "unsymmetric_pattern", "far"])
def test_native_fast_path_agrees_with_the_general_path(case):
    """api._prepare checks a canonical real CSR matrix with the native hsg_csr_inspect (host threads);
    every input must come out as the general path (_as_csr + _hermitian_check) makes it: the same
    matrix, the same defect, the same error."""
    m = _sym(300, 0.02, 11)
    if case == "near":
        noise = m.copy()
        noise.data = noise.data * (1e-13 * np.random.default_rng(12).standard_normal(noise.nnz))
        m = (m + noise).tocsr()
    elif case == "upper_only":
        m = sp.triu(m, format="csr")
    elif case == "zeros":
        m = m.copy()
        m.data[3] = 0.0
    elif case == "unsorted":
        m = m.copy()
        m.indices[:2] = m.indices[:2][::-1].copy()
        m.has_sorted_indices = False
    elif case == "unsymmetric_pattern":
        m = m.tolil()
        m[0, 7] = 1e-14
        m[7, 0] = 0.0
        m = m.tocsr()
        m.eliminate_zeros()
    elif case == "far":
        m = m.tolil()
        m[2, 9] = m[2, 9] + 1.0
        m = m.tocsr()
    original = m.copy()
    try:
        want, want_d = api._hermitian_check(api._as_csr(m.copy(), "A", "auto"), "A", 1e-10)
    except NotHermitianError:
        with pytest.raises(NotHermitianError):
            api._prepare(m, "A", "auto", 1e-10)
        return
    got, got_d = api._prepare(m, "A", "auto", 1e-10)
    _same(got, want)
    assert abs(got_d - want_d) <= 1e-12 * max(want_d, 1e-300)
    _same(m, original)  # the caller's matrix is not modified
