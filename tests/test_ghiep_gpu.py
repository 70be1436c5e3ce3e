"""GPU parity of the GHIEP path (B indefinite; hsolve src/driver/indefinite.cpp solve_indefinite):
the reference's waveguide-50ghz example against its dense spectrum (tests/golden/waveguide.npz =
hsolve examples/cases + refs/waveguide-50ghz), and a congruence-transformed block pencil with known
complex eigenvalues. Eigenvalues within 1e-10 relative, every backward error <= tol, no certificate."""
import numpy as np
import pytest
import scipy.sparse as sp

import hsolve_b200 as hsolve
from hsolve_b200.errors import UnsupportedError

pytestmark = pytest.mark.gpu

EIG_RTOL = 1e-10
WAVEGUIDE_SIGMA = -0.5013049800407187  # examples/cases/waveguide-50ghz/config.json in hsolve


def _waveguide(golden):
    z = np.load(golden / "waveguide.npz")
    n = z["A_indptr"].size - 1
    a = sp.csr_matrix((z["A_data"], z["A_indices"], z["A_indptr"]), shape=(n, n))
    b = sp.csr_matrix((z["B_data"], z["B_indices"], z["B_indptr"]), shape=(n, n))
    return a, b, np.real(z["eigenvalues"])


def _eta(a, b, lam, x):
    na = np.linalg.norm(a.toarray(), 2)
    nb = np.linalg.norm(b.toarray(), 2)
    r = a @ x - lam * (b @ x)
    return np.linalg.norm(r) / ((na + abs(lam) * nb) * np.linalg.norm(x))


def test_waveguide_nearest_18(golden):
    a, b, w = _waveguide(golden)
    res = hsolve.solve(a, b, sigma=WAVEGUIDE_SIGMA, k=18)
    rep = res.report
    assert rep["problem"] == "GHIEP" and rep["method"] == "shift_invert_krylov_schur"
    assert res.success, rep
    assert not rep["certificate"]["performed"]
    assert res.complex_eigenvalues.size == 0
    order = np.argsort(np.abs(w - WAVEGUIDE_SIGMA), kind="stable")
    want = np.sort(w[order[:18]])
    assert (want < 0).all()  # the 18 propagating modes, clear of the 64-fold zero cluster
    np.testing.assert_allclose(np.sort(res.eigenvalues), want, rtol=EIG_RTOL)
    # nearest first, unit 2-norm vectors, independent within the double eigenvalue
    d = np.abs(res.eigenvalues - WAVEGUIDE_SIGMA)
    assert (np.diff(d) >= -1e-12).all()
    x = res.eigenvectors
    np.testing.assert_allclose(np.linalg.norm(x, axis=0), 1.0, rtol=1e-12)
    assert np.linalg.matrix_rank(x, tol=1e-6) == 18
    for q in range(18):
        assert rep["pairs"][q]["backward_error"] <= 1e-10
        assert _eta(a, b, res.eigenvalues[q], x[:, q]) <= 1e-10


def _complex_pencil(seed=7):
    """A block pencil (2 x 2 blocks with B = diag(1, -1) and complex eigenvalue pairs, 1 x 1 blocks
    with B = +-1) under the congruence P^T (.) P with P = I + 0.3 (superdiagonal): eigenvalues known."""
    rng = np.random.default_rng(seed)
    q, r = 30, 60
    n = 2 * q + r
    ra, rb = [], []
    lam = []
    for i in range(q):
        re, im = rng.uniform(-1.0, 1.0), rng.uniform(0.01, 0.15)
        # lambda = ((a - c) +- sqrt((a + c)^2 - 4 b^2)) / 2 with a + c = s, b > |s| / 2
        s = rng.uniform(-0.5, 0.5)
        av, cv = (2 * re + s) / 2, (s - 2 * re) / 2
        bv = np.sqrt(s * s + 4 * im * im) / 2
        ra.append(np.array([[av, bv], [bv, cv]]))
        rb.append(np.diag([1.0, -1.0]))
        lam += [complex(re, im), complex(re, -im)]
    for j in range(r):
        d, sg = rng.uniform(-3.0, 3.0), rng.choice([-1.0, 1.0])
        ra.append(np.array([[sg * d]]))
        rb.append(np.array([[sg]]))
        lam.append(complex(d, 0.0))
    a0 = sp.block_diag([sp.csr_matrix(m) for m in ra], format="csr")
    b0 = sp.block_diag([sp.csr_matrix(m) for m in rb], format="csr")
    p = sp.eye(n, format="csr") + 0.3 * sp.eye(n, k=1, format="csr")
    a = (p.T @ a0 @ p).tocsr()
    b = (p.T @ b0 @ p).tocsr()
    return a, b, np.array(lam)


def test_complex_pairs_nearest():
    a, b, lam = _complex_pencil()
    sigma = 0.137
    d = np.abs(lam - sigma)
    order = np.argsort(d, kind="stable")
    ds = d[order]
    k = next(k for k in range(12, 30) if ds[k] - ds[k - 1] > 1e-3)  # no pair split, no tie
    want = lam[order[:k]]
    res = hsolve.solve(a, b, sigma=sigma, k=k)
    assert res.report["problem"] == "GHIEP"
    assert res.success, res.report
    got_c = res.complex_eigenvalues
    want_c = want[np.abs(want.imag) > 1e-8]
    want_r = np.sort(want[np.abs(want.imag) <= 1e-8].real)
    assert got_c.size == want_c.size and got_c.size > 0
    np.testing.assert_allclose(np.sort(res.eigenvalues), want_r, rtol=EIG_RTOL)
    key = lambda z: (round(z.real, 6), round(z.imag, 6))  # noqa: E731
    gs, ws = sorted(got_c, key=key), sorted(want_c, key=key)
    for g, e in zip(gs, ws):
        assert abs(g - e) <= EIG_RTOL * abs(e)
    # the report lists the real pairs, then the complex ones, every one accepted
    pr = res.report["pairs"]
    assert len(pr) == k
    assert all(p["lambda_im"] == 0.0 for p in pr[: res.eigenvalues.size])
    assert all(p["lambda_im"] != 0.0 for p in pr[res.eigenvalues.size:])
    assert all(p["backward_error"] <= 1e-10 for p in pr)
    for j in range(got_c.size):
        assert _eta(a, b, got_c[j], res.complex_eigenvectors[:, j]) <= 1e-10


def test_ghiep_session_and_targets(golden):
    a, b, w = _waveguide(golden)
    s = hsolve.Session(a, b)
    r1 = s.solve(sigma=WAVEGUIDE_SIGMA, k=18)
    r2 = s.solve(sigma=WAVEGUIDE_SIGMA, k=18)
    np.testing.assert_allclose(r1.eigenvalues, r2.eigenvalues, rtol=1e-12)
    # a smaller k around another shift among the modes
    r3 = s.solve(sigma=-0.7, k=4)
    order = np.argsort(np.abs(w + 0.7), kind="stable")
    np.testing.assert_allclose(np.sort(r3.eigenvalues), np.sort(w[order[:4]]), rtol=EIG_RTOL)
    with pytest.raises(UnsupportedError):
        s.solve(lower=-1.0, upper=-0.5, mode="interval")
