"""CPU: the host dense routines of the Krylov driver (hsolve_b200/csrc/dense_host.cpp: the symmetric
eigensolver of Rayleigh-Ritz, the Cholesky / triangular inverse of CholQR, the small products),
compiled from the product source into a test harness and checked against numpy, including the
clustered and exactly degenerate spectra that the PEC cavities produce.
"""
import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "hsolve_b200" / "csrc"

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("dense") / "libdense_harness.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", f"-I{SRC}", str(SRC / "dense_host.cpp"),
                    str(Path(__file__).with_name("dense_host_harness.cpp")), "-o", str(out)], check=True)
    L = ctypes.CDLL(str(out))
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.t_sym_eig.argtypes = [I, P, P, P]
    L.t_sym_eig.restype = I
    L.t_cholesky.argtypes = [I, P, D, P]
    L.t_cholesky.restype = I
    L.t_lower_inverse.argtypes = [I, P, P]
    L.t_matmul.argtypes = [I, I, I, P, P, P]
    L.t_schur.argtypes = [I, P, P, I, D, P, P, P]
    L.t_schur.restype = I
    L.t_pivoted_basis.argtypes = [I, I, P, I, D, P]
    L.t_pivoted_basis.restype = I
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _eig(lib, a):
    n = a.shape[0]
    a = np.asfortranarray(a, dtype=np.float64)
    w = np.zeros(n)
    v = np.zeros((n, n), order="F")
    assert lib.t_sym_eig(n, _p(a), _p(w), _p(v)) == 0
    return w, v


def _check_eig(lib, a):
    n = a.shape[0]
    w, v = _eig(lib, a)
    full = np.tril(a) + np.tril(a, -1).T
    scale = max(np.abs(np.linalg.eigvalsh(full)).max(), 1e-300) if n else 1.0
    assert np.all(np.diff(w) >= 0)
    np.testing.assert_allclose(w, np.linalg.eigvalsh(full), rtol=0, atol=1e-13 * scale * max(1, n) ** 0.5)
    assert np.abs(full @ v - v * w).max() <= 1e-12 * scale * max(1, n) ** 0.5
    assert np.abs(v.T @ v - np.eye(n)).max() <= 1e-12 * max(1, n)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 17, 40, 96, 128])
def test_sym_eig_random(lib, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n))
    _check_eig(lib, x + x.T)


def test_sym_eig_reads_the_lower_triangle(lib):
    rng = np.random.default_rng(5)
    x = rng.standard_normal((30, 30))
    a = x + x.T
    garbage = np.triu(rng.standard_normal((30, 30)) * 1e6, 1)
    w1, _ = _eig(lib, a)
    w2, _ = _eig(lib, np.tril(a) + garbage)
    np.testing.assert_array_equal(w1, w2)


@pytest.mark.parametrize("mults", [(2, 2, 2, 3), (3, 6, 12), (1, 1, 40), (12, 12, 12, 1)])
def test_sym_eig_degenerate_clusters(lib, mults):
    rng = np.random.default_rng(sum(mults))
    levels = np.repeat(np.arange(1, len(mults) + 1, dtype=float) * 7.5, mults)
    n = levels.size
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    a = (q * levels) @ q.T
    a = 0.5 * (a + a.T)
    _check_eig(lib, a)
    # split clusters at rounding level, as a Krylov projection of a degenerate level produces
    b = a + 1e-14 * np.diag(rng.standard_normal(n))
    _check_eig(lib, 0.5 * (b + b.T))


def test_sym_eig_special(lib):
    _check_eig(lib, np.zeros((6, 6)))
    _check_eig(lib, np.diag([3.0, -1.0, 2.0, 2.0, 0.0]))
    t = np.diag(np.full(20, 2.0)) + np.diag(np.full(19, -1.0), 1) + np.diag(np.full(19, -1.0), -1)
    w, _ = _eig(lib, t)
    exact = 2.0 - 2.0 * np.cos(np.pi * np.arange(1, 21) / 21)
    np.testing.assert_allclose(w, exact, rtol=0, atol=1e-14)


def test_cholesky_and_lower_inverse(lib):
    rng = np.random.default_rng(11)
    for p in (1, 4, 8, 16):
        x = rng.standard_normal((p, p + 3))
        g = np.asfortranarray(x @ x.T)
        l = np.zeros((p, p), order="F")
        assert lib.t_cholesky(p, _p(g), 0.0, _p(l)) == 1
        assert np.allclose(np.triu(l, 1), 0)
        np.testing.assert_allclose(l @ l.T, g, rtol=1e-13, atol=1e-13 * np.abs(g).max())
        inv = np.zeros((p, p), order="F")
        lib.t_lower_inverse(p, _p(l), _p(inv))
        np.testing.assert_allclose(inv @ l, np.eye(p), atol=1e-12)
    bad = np.asfortranarray(np.diag([1.0, -1.0, 2.0]))
    l = np.zeros((3, 3), order="F")
    assert lib.t_cholesky(3, _p(bad), 0.0, _p(l)) == 0
    near = np.asfortranarray(np.diag([1.0, 1e-14, 2.0]))
    assert lib.t_cholesky(3, _p(near), 0.0, _p(l)) == 1
    assert lib.t_cholesky(3, _p(near), 1e-12, _p(l)) == 0   # rel_tol rejects the tiny pivot


def test_matmul(lib):
    rng = np.random.default_rng(12)
    for m, k, n in [(1, 1, 1), (7, 3, 5), (40, 16, 24)]:
        a = np.asfortranarray(rng.standard_normal((m, k)))
        b = np.asfortranarray(rng.standard_normal((k, n)))
        b[0, 0] = 0.0
        c = np.zeros((m, n), order="F")
        lib.t_matmul(m, k, n, _p(a), _p(b), _p(c))
        np.testing.assert_allclose(c, a @ b, rtol=1e-14, atol=1e-13)


def _schur(lib, a, count, sort=True, cluster_rtol=1e-8):
    n = a.shape[0]
    af = np.asfortranarray(a, dtype=np.float64)
    t = np.zeros((n, n), dtype=np.complex128, order="F")
    u = np.zeros((n, n), dtype=np.complex128, order="F")
    y = np.zeros((n, count), dtype=np.complex128, order="F")
    key = np.zeros(n) if sort else None
    rc = lib.t_schur(n, _p(af), None if key is None else _p(key), count, cluster_rtol, _p(t), _p(u), _p(y))
    assert rc == 0
    return t, u, y


@pytest.mark.parametrize("n,seed", [(1, 0), (2, 1), (7, 2), (40, 3), (120, 4)])
def test_complex_schur_of_random_matrices(lib, n, seed):
    a = np.random.default_rng(seed).standard_normal((n, n))
    t, u, y = _schur(lib, a, n)
    assert np.abs(u.conj().T @ u - np.eye(n)).max() < 1e-12
    assert np.abs(np.tril(t, -1)).max(initial=0.0) == 0.0
    assert np.abs(u @ t @ u.conj().T - a).max() < 1e-12 * max(1.0, np.abs(a).max()) * n
    lam = np.diag(t)
    ref = np.linalg.eigvals(a)
    assert np.all(np.diff(np.abs(lam)) <= 1e-12 * np.abs(lam).max())  # sorted by magnitude, largest first
    for z in ref:
        assert np.min(np.abs(lam - z)) <= 1e-9 * max(1.0, np.abs(ref).max())
    x = u @ y
    for k in range(n):
        assert np.linalg.norm(a @ x[:, k] - lam[k] * x[:, k]) <= 1e-9 * max(1.0, np.abs(a).max()) * np.sqrt(n)


def test_schur_eigenvectors_of_a_multiple_eigenvalue_are_independent(lib):
    """A diagonalizable matrix with triple and double real eigenvalues and a complex pair: the
    vectors of each multiple eigenvalue span its eigenspace."""
    rng = np.random.default_rng(7)
    d = np.array([5.0, 5.0, 5.0, -2.0, -2.0, 0.5, 0.1])
    blk = np.diag(d)
    blk[5:7, 5:7] = [[0.5, 1.0], [-1.0, 0.5]]  # eigenvalues 0.5 +- i
    s = rng.standard_normal((7, 7))
    a = s @ blk @ np.linalg.inv(s)
    t, u, y = _schur(lib, a, 7, cluster_rtol=1e-7)
    lam = np.diag(t)
    x = u @ y
    for k in range(7):
        assert np.linalg.norm(a @ x[:, k] - lam[k] * x[:, k]) < 1e-8
    for value, mult in ((5.0, 3), (-2.0, 2)):
        idx = np.flatnonzero(np.abs(lam - value) < 1e-6)
        assert idx.size == mult
        assert np.linalg.matrix_rank(x[:, idx], tol=1e-6) == mult


def test_pivoted_basis_takes_genuine_directions_before_rounding_noise(lib):
    """The real basis of a double real eigenvalue's eigenspace from complex Ritz vectors: each is a
    phase times a real eigenvector plus noise, so its imaginary part after the phase is mostly noise;
    the greedy basis must span the two true directions and ignore the noise."""
    rng = np.random.default_rng(5)
    m = 30
    u, _ = np.linalg.qr(rng.standard_normal((m, 2)))
    noise = 1e-9 * rng.standard_normal((m, 4))
    c1 = np.exp(0.3j) * u[:, 0] + noise[:, 0] + 1j * noise[:, 1]
    c2 = np.exp(-1.1j) * (0.6 * u[:, 0] + 0.8 * u[:, 1]) + noise[:, 2] + 1j * noise[:, 3]
    # pool: the two imaginary-part noise directions first, then the real and imaginary parts
    pool = np.column_stack([noise[:, 1] / 1e-9 * 1e-9, c1.real, c1.imag, c2.real, c2.imag])
    pool = np.asfortranarray(pool)
    q = np.zeros((m, 2), order="F")
    r = lib.t_pivoted_basis(m, pool.shape[1], _p(pool), 2, 1e-3, _p(q))
    assert r == 2
    assert np.abs(q.T @ q - np.eye(2)).max() < 1e-12
    # q spans span(u): the projection of u on q is complete
    assert np.linalg.norm(u - q @ (q.T @ u)) < 1e-7
    # a pool of one genuine direction yields one column
    pool1 = np.asfortranarray(np.column_stack([u[:, 0], 1e-10 * rng.standard_normal(m)]))
    assert lib.t_pivoted_basis(m, 2, _p(pool1), 2, 1e-3, _p(q)) == 1
