"""Randomized exclusion certificate on the GPU (hsolve's exclusion_check, include/hsolve/verify.hpp:
18-80) on a Yee/FIT cavity whose spectrum is known exactly: the found nearest eigenvectors pass, the
same set with one vector withheld is detected, and a gap too narrow for the plan's budget is
inconclusive."""
import numpy as np
import pytest

import hsolve_b200 as hsolve
from hsolve_b200.gen import yee
from oracle import yee_exact

pytestmark = pytest.mark.gpu


def _setup():
    box = yee.Box((14, 11, 8), (1.0, 0.75, 0.55))
    a, b = yee.pencil(box, "generalized")
    w = yee_exact.exact_spectrum(box.cells, box.lengths)
    sigma = 150.0
    d = np.sort(np.abs(w - sigma))
    # the first K >= 6 whose next distance is at least 20 % larger: no cluster straddles the radius
    k = next(k for k in range(6, 30) if d[k] > 1.2 * d[k - 1])
    sess = hsolve.Session(a, b)
    res = sess.solve(sigma=sigma, k=k)
    assert res.report["success"]
    return sess, res, sigma, d, k


def test_exclusion_passes_detects_and_refuses():
    sess, res, sigma, d, k = _setup()
    x = res.eigenvectors
    lam = res.eigenvalues
    assert x.shape[1] == k
    np.testing.assert_allclose(np.sort(np.abs(lam - sigma)), d[:k], rtol=1e-9)
    radius = d[k - 1] * (1.0 + 1e-6)
    pass_radius = d[k - 1] + 0.9 * (d[k] - d[k - 1])
    r = sess.exclusion_check(x, sigma=sigma, radius=radius, pass_radius=pass_radius, delta=1e-12)
    assert r["status"] == "passed", r
    assert r["found_inside"] == k and r["certified_inside"] == k and r["deflated"] == k
    assert r["coupling"] < 1e-6 / radius
    assert r["failure_probability"] <= 1e-12 or r["exact"]
    assert r["block_steps"] == r["block_steps_planned"]
    assert r["op_applications"] == k + r["block_steps"] * r["block_size"]
    assert r["max_ritz"] < 1.0 / pass_radius
    assert r["new_count"] == 0 and r["rigorous"]
    # the nearest eigenvector withheld: the run on the complement finds its eigenvalue
    j0 = int(np.argmin(np.abs(lam - sigma)))
    x2 = np.delete(x, j0, axis=1)
    r2 = sess.exclusion_check(x2, sigma=sigma, radius=radius, pass_radius=pass_radius, delta=1e-12)
    assert r2["status"] == "detected", r2
    assert r2["found_inside"] == k - 1 and r2["new_inside"] >= 1
    assert r2["max_ritz"] == pytest.approx(1.0 / d[0], rel=1e-4)
    # a pass radius barely above the radius: the plan exceeds the budget, no statement, no run
    r3 = sess.exclusion_check(x, sigma=sigma, radius=radius, pass_radius=radius * (1.0 + 1e-9), delta=1e-12)
    assert r3["status"] == "inconclusive" and r3["block_steps"] == 0
    with pytest.raises(hsolve.InvalidInputError):
        sess.exclusion_check(x, sigma=sigma, radius=radius, pass_radius=radius)
    sess.close()


def test_exclusion_complex_pencil_runs_on_the_embedding():
    """A complex Hermitian (Bloch) pencil: the found complex eigenvectors are embedded into the real
    2n problem the session holds, where every eigenvalue appears twice; the found set passes with
    every count doubled."""
    box = yee.Box((7, 6, 6), (1.0, 0.9, 0.8), "bloch", (0.9, 0.4, 0.2))
    a, b = yee.pencil(box, "generalized")
    w = yee_exact.exact_spectrum(box.cells, box.lengths, "bloch", box.phases)
    wp = np.sort(w[w > 1.0])
    sigma = 0.5 * (wp[8] + wp[9]) + 0.123
    d = np.sort(np.abs(w - sigma))
    k = next(k for k in range(4, 30) if d[k] > 1.2 * d[k - 1])
    sess = hsolve.Session(a, b)
    res = sess.solve(sigma=sigma, k=k)
    assert res.report["success"]
    x = res.eigenvectors
    assert np.iscomplexobj(x) and x.shape[1] == k
    radius = d[k - 1] * (1.0 + 1e-6)
    pass_radius = d[k - 1] + 0.9 * (d[k] - d[k - 1])
    r = sess.exclusion_check(x, sigma=sigma, radius=radius, pass_radius=pass_radius, delta=1e-12)
    assert r["status"] == "passed", r
    assert r["deflated"] == 2 * k and r["found_inside"] == 2 * k and r["certified_inside"] == 2 * k
    assert r["dimension"] == 2 * a.shape[0] - 2 * k
    assert r["failure_probability"] <= 1e-12 or r["exact"]
    sess.close()
