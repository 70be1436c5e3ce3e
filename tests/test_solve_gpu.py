"""GPU end-to-end parity of hsolve_b200.solve against the reference's example cases (rebuilt by the
generator, spectra from tests/golden/examples.json = hsolve examples/refs/*) and exact Yee spectra:
eigenvalues within 1e-10 relative, every backward error <= tol, certificate counts equal to the
exact counts #{lambda in window}."""
import json

import numpy as np
import pytest
import scipy.sparse as sp

import hsolve_b200 as hsolve
from hsolve_b200.gen import yee
from oracle import yee_exact

pytestmark = pytest.mark.gpu

EIG_RTOL = 1e-10


def _example(golden, name):
    e = json.loads((golden / "examples.json").read_text())[name]
    p = e["meta"]["params"]
    box = yee.Box(tuple(p["cells"]), tuple(p["lengths"]), p["boundary"], tuple(p["phases"]))
    a, b = yee.pencil(box, p["form"])
    return e, box, a, b


def _check_pairs(res, tol=1e-10):
    assert res.success, res.report
    for pr in res.report["pairs"]:
        assert pr["backward_error"] <= tol, pr


def test_nearest_multiplicity_example(golden):
    e, box, a, b = _example(golden, "pec-cavity-multiplicity")
    t = e["config"]["target"]
    res = hsolve.solve(a, b, sigma=t["sigma"], k=t["k"])
    _check_pairs(res)
    ref = np.array(e["ref_nearest"])
    order = np.argsort(np.abs(ref - t["sigma"]), kind="stable")
    want = np.sort(ref[order[: t["k"]]])
    np.testing.assert_allclose(np.sort(res.eigenvalues), want, rtol=EIG_RTOL)
    c = res.report["certificate"]
    w = yee_exact.exact_spectrum(box.cells, box.lengths)
    assert c["passed"] and c["method"] == "exact"
    assert c["count_inertia"] == yee_exact.count_below(w, c["upper"]) - yee_exact.count_below(w, c["lower"])
    # B-orthonormal eigenvectors
    x = res.eigenvectors
    assert np.abs(x.T @ x - np.eye(x.shape[1])).max() < 1e-10


def test_interval_slicing_example(golden):
    e, box, a, b = _example(golden, "interval-slicing")
    t = e["config"]["target"]
    res = hsolve.solve(a, b, lower=t["lower"], upper=t["upper"])
    _check_pairs(res)
    ref = np.sort(np.array(e["ref_interval"]))
    assert res.eigenvalues.size == ref.size
    np.testing.assert_allclose(res.eigenvalues, ref, rtol=EIG_RTOL)
    assert res.report["certificate"]["count_inertia"] == ref.size


def test_interval_many_slices(golden):
    """A window holding several slices: cut counts certify each slice."""
    box = yee.Box((12, 12, 12))
    a, _ = yee.pencil(box)
    w = yee_exact.exact_spectrum(box.cells)
    lo, hi = yee_exact.mid_gap_shifts(w, 30, 1e-6)[17], yee_exact.mid_gap_shifts(w, 30, 1e-6)[19]
    res = hsolve.solve(a, lower=lo, upper=hi, config={"slice_size": 40})
    _check_pairs(res)
    want = w[(w >= lo) & (w <= hi)]
    assert len(res.report["slices"]) >= 2
    np.testing.assert_allclose(res.eigenvalues, want, rtol=EIG_RTOL)


def test_generalized_lowfreq_window(golden):
    e, box, a, b = _example(golden, "lowfreq-null-space")
    t = e["config"]["target"]
    res = hsolve.solve(a, b, lower=t["lower"], upper=t["upper"])
    _check_pairs(res)
    np.testing.assert_allclose(res.eigenvalues, np.sort(e["ref_interval"]), rtol=EIG_RTOL)
    x = res.eigenvectors
    assert np.abs(x.T @ (b @ x) - np.eye(x.shape[1])).max() < 1e-10


def test_near_singular_shift_example(golden):
    e = json.loads((golden / "examples.json").read_text())["near-singular-shift"]
    z = np.load(golden / "near_singular.npz")
    a = sp.csr_matrix((z["data"], z["indices"], z["indptr"]))
    t = e["config"]["target"]
    res = hsolve.solve(a, sigma=t["sigma"], k=t["k"])
    _check_pairs(res)
    ref = np.array(e["ref_nearest"])
    order = np.argsort(np.abs(ref - t["sigma"]), kind="stable")
    np.testing.assert_allclose(np.sort(res.eigenvalues), np.sort(ref[order[: t["k"]]]), rtol=EIG_RTOL)
    assert res.report["shift_retries"] >= 1


def test_generalized_nearest_box():
    box = yee.Box((14, 11, 8), (1.0, 0.75, 0.55))
    a, b = yee.pencil(box, "generalized")
    w = yee_exact.exact_spectrum(box.cells, box.lengths)
    sigma = 150.0
    res = hsolve.solve(a, b, sigma=sigma, k=10)
    _check_pairs(res)
    order = np.argsort(np.abs(w - sigma), kind="stable")
    np.testing.assert_allclose(np.sort(res.eigenvalues), np.sort(w[order[:10]]), rtol=EIG_RTOL)


def test_errors_follow_reference_classes():
    a = sp.random(20, 20, density=0.3, random_state=1).tocsr()
    with pytest.raises(hsolve.NotHermitianError):
        hsolve.solve(a + sp.identity(20), sigma=0.1, k=2, storage="full")
    with pytest.raises(hsolve.InvalidInputError):
        hsolve.solve(sp.identity(5), sigma=0.0, k=2, config={"no_such_key": 1})


def test_bloch_cell_complex_example(golden):
    """hsolve examples/bloch-cell-complex: a complex Hermitian Bloch cell, solved through the real
    2n embedding; eigenvalues match the reference's stored spectrum and the vectors come back
    complex and orthonormal."""
    e, box, a, b = _example(golden, "bloch-cell-complex")
    assert np.iscomplexobj(a.data)
    t = e["config"]["target"]
    res = hsolve.solve(a, b, sigma=t["sigma"], k=t["k"])
    _check_pairs(res)
    assert res.report["complex_scalars"] and res.eigenvectors.dtype == np.complex128
    ref = np.array(e["ref_nearest"])
    want = np.sort(ref[np.argsort(np.abs(ref - t["sigma"]), kind="stable")[: t["k"]]])
    np.testing.assert_allclose(np.sort(res.eigenvalues), want, rtol=EIG_RTOL)
    x = res.eigenvectors
    np.testing.assert_allclose(x.conj().T @ x, np.eye(x.shape[1]), atol=1e-10)
    cert = res.report["certificate"]
    w = yee_exact.exact_spectrum(box.cells, box.lengths, "bloch", box.phases)
    assert cert["passed"] and cert["count_inertia"] == cert["count_found"]
    assert cert["count_inertia"] == yee_exact.count_below(w, cert["upper"]) - yee_exact.count_below(w, cert["lower"])


def test_bloch_cell_complex_interval_exact_spectrum():
    box = yee.Box((8, 7, 6), (1.0, 0.9, 0.8), "bloch", (0.4 * np.pi, 0.25 * np.pi, 0.1 * np.pi))
    a, b = yee.pencil(box, "generalized")
    w = yee_exact.exact_spectrum(box.cells, box.lengths, "bloch", box.phases)
    cuts = yee_exact.mid_gap_shifts(w[w > 1.0], 12, 1e-6)
    lo, hi = cuts[3], cuts[9]
    sess = hsolve.Session(a, b)
    for _ in range(2):
        res = sess.solve(lower=lo, upper=hi)
        _check_pairs(res)
        want = w[(w >= lo) & (w <= hi)]
        np.testing.assert_allclose(res.eigenvalues, want, rtol=EIG_RTOL)
        assert res.report["certificate"]["count_inertia"] == want.size
        x = res.eigenvectors
        np.testing.assert_allclose(x.conj().T @ (b @ x), np.eye(want.size), atol=1e-10)


def test_complex_dtype_with_real_values_returns_complex_vectors():
    a, _ = yee.pencil(yee.Box((6, 5, 4)))
    res = hsolve.solve(a.astype(np.complex128), sigma=30.0, k=4)
    _check_pairs(res)
    assert res.eigenvectors.dtype == np.complex128 and not res.report["complex_scalars"]


def test_repeated_pattern_reuses_analysis_with_new_values():
    """Solves on one sparsity pattern reuse the cached nested-dissection analysis; new values on
    that pattern (here 2A) still give the right certified eigenpairs."""
    box = yee.Box((10, 9, 8))
    a, _ = yee.pencil(box)
    w = yee_exact.exact_spectrum(box.cells)
    cuts = yee_exact.mid_gap_shifts(w[w > 1.0], 10, 1e-6)
    lo, hi = cuts[2], cuts[5]
    r1 = hsolve.solve(a, lower=lo, upper=hi)
    r2 = hsolve.solve(2.0 * a, lower=2.0 * lo, upper=2.0 * hi)
    _check_pairs(r1)
    _check_pairs(r2)
    want = w[(w >= lo) & (w <= hi)]
    np.testing.assert_allclose(r1.eigenvalues, want, rtol=EIG_RTOL)
    np.testing.assert_allclose(r2.eigenvalues, 2.0 * want, rtol=EIG_RTOL)
    assert r2.report["factor_stats"]["ordering_s"] == 0.0  # the second call found the analysis cached


def test_server_runs_mixed_requests_concurrently():
    """The request-stream server: real and complex pencils of different sizes, admitted by device
    memory and solved concurrently, each certified and equal to its exact spectrum."""
    from hsolve_b200.serve import Server

    cases = []
    for cells, boundary, phases in [((8, 7, 6), "pec", (0.0, 0.0, 0.0)), ((7, 6, 6), "bloch", (0.9, 0.4, 0.2)),
                                    ((9, 8, 7), "pec", (0.0, 0.0, 0.0)), ((7, 6, 6), "bloch", (1.3, 0.7, 0.1))]:
        box = yee.Box(cells, (1.0, 0.9, 0.8), boundary, phases)
        a, b = yee.pencil(box, "generalized")
        w = yee_exact.exact_spectrum(box.cells, box.lengths, boundary, box.phases)
        cuts = yee_exact.mid_gap_shifts(w[w > 1.0], 8, 1e-6)
        cases.append((a, b, cuts[1], cuts[6], w))
    with Server(workers=2) as srv:
        futs = [srv.submit(a, b, lower=lo, upper=hi) for a, b, lo, hi, _ in cases]
        results = [f.result() for f in futs]
    for (a, b, lo, hi, w), res in zip(cases, results):
        _check_pairs(res)
        np.testing.assert_allclose(res.eigenvalues, w[(w >= lo) & (w <= hi)], rtol=EIG_RTOL)
    st = srv.stats()
    assert st["requests"] == 4 and st["certified"] == 4 and not st["failed"]
    assert st["latency_p99_s"] >= st["latency_p50_s"] > 0


def test_dealer_parts_of_one_window_compose_to_the_exact_spectrum():
    """hsolve_b200.parallel on one GPU: the window cut into three parts by FP64 counts, each part a
    certified solve of its own, the gathered result equal to the exact spectrum of the whole window."""
    from hsolve_b200.parallel import Dealer

    box = yee.Box((12, 11, 10), (1.0, 0.75, 0.55))
    a, b = yee.pencil(box, "generalized")
    w = yee_exact.exact_spectrum(box.cells, box.lengths)
    lo, hi = 40.0, 200.0
    with Dealer() as d:
        lam, vec, rep = d.solve_interval(a, b, lo, hi, parts=3)
    want = w[(w >= lo) & (w < hi)]
    assert rep["passed"] and len(rep["parts"]) == 3 and rep["count_inertia"] == want.size
    np.testing.assert_allclose(lam, want, rtol=EIG_RTOL)
    assert np.abs(vec.T @ (b @ vec) - np.eye(want.size)).max() < 1e-10


def test_server_results_are_the_same_alone_and_in_the_mix():
    """Continuous batching must not change results: every request solved alone (one worker, one
    request at a time) and again in a mixed stream of real and complex pencils of different sizes
    (three workers, all submitted at once) gives the same certified eigenvalues (within 1e-10
    relative) and the same certificate counts."""
    from hsolve_b200.serve import Server

    reqs = []
    for cells, boundary, phases in [((8, 7, 6), "pec", (0.0, 0.0, 0.0)), ((7, 6, 6), "bloch", (0.9, 0.4, 0.2)),
                                    ((10, 9, 8), "pec", (0.0, 0.0, 0.0)), ((6, 6, 6), "bloch", (1.3, 0.7, 0.1)),
                                    ((9, 8, 7), "pec", (0.0, 0.0, 0.0))]:
        box = yee.Box(cells, (1.0, 0.9, 0.8), boundary, phases)
        a, b = yee.pencil(box, "generalized")
        w = yee_exact.exact_spectrum(box.cells, box.lengths, boundary, box.phases)
        cuts = yee_exact.mid_gap_shifts(w[w > 1.0], 8, 1e-6)
        reqs.append((a, b, dict(lower=cuts[1], upper=cuts[6])))
    alone = []
    with Server(workers=1) as srv:
        for a, b, t in reqs:
            alone.append(srv.submit(a, b, **t).result())
    with Server(workers=3) as srv:
        futs = [srv.submit(a, b, **t) for a, b, t in reqs]
        mixed = [f.result() for f in futs]
    for r1, r2 in zip(alone, mixed):
        _check_pairs(r1)
        _check_pairs(r2)
        assert r1.eigenvalues.size == r2.eigenvalues.size > 0
        np.testing.assert_allclose(r2.eigenvalues, r1.eigenvalues, rtol=EIG_RTOL)
        c1, c2 = r1.report["certificate"], r2.report["certificate"]
        assert c1["count_inertia"] == c2["count_inertia"] and c1["passed"] and c2["passed"]


def test_registered_pencil_served_concurrently_matches_alone():
    """A registered (resident) pencil served by four workers at once, every request with its own
    Krylov seed and target: each result equals the same request solved alone on a session, and the
    intervals match the exact spectrum."""
    from hsolve_b200.serve import Server

    box = yee.Box((12, 11, 10), (1.0, 0.75, 0.55))
    a, b = yee.pencil(box, "generalized")
    w = yee_exact.exact_spectrum(box.cells, box.lengths)
    cuts = yee_exact.mid_gap_shifts(w[(w > 1.0) & (w < 600.0)], 40, 1e-6)
    targets = [dict(lower=cuts[i], upper=cuts[i + 6], config={"seed": 100 + i}) for i in range(0, 24, 3)]
    with Server(workers=4) as srv:
        h = srv.register(a, b)
        futs = [srv.submit(pencil=h, **t) for t in targets]
        served = [f.result() for f in futs]
    s = hsolve.Session(a, b)
    for t, r in zip(targets, served):
        _check_pairs(r)
        alone = s.solve(**t)
        want = w[(w >= t["lower"]) & (w < t["upper"])]
        np.testing.assert_allclose(r.eigenvalues, want, rtol=EIG_RTOL)
        np.testing.assert_allclose(r.eigenvalues, alone.eigenvalues, rtol=EIG_RTOL)
        assert r.report["certificate"]["count_inertia"] == want.size
    s.close()


def test_concurrent_sessions_nearest_and_interval_stay_exact():
    """Four threads, each with its own session on the same pencil, alternate nearest and interval
    targets back to back: buffers that one request releases while its last kernels are still
    queued are reused by the others only after those kernels ran, so every result stays equal to
    the exact spectrum."""
    import threading

    box = yee.Box((11, 10, 9), (1.0, 0.85, 0.7))
    a, b = yee.pencil(box, "generalized")
    w = yee_exact.exact_spectrum(box.cells, box.lengths)
    wl = w[(w > 1.0) & (w < 500.0)]
    cuts = yee_exact.mid_gap_shifts(wl, 24, 1e-6)
    errors = []

    def worker(t):
        s = hsolve.Session(a, b)
        try:
            for i in range(6):
                q = (4 * t + i) % (len(cuts) - 4)
                if i % 2:
                    r = s.solve(lower=cuts[q], upper=cuts[q + 3], config={"seed": 10 * t + i})
                    want = w[(w >= cuts[q]) & (w < cuts[q + 3])]
                    got = r.eigenvalues
                else:
                    sigma = cuts[q] + 0.3 * (cuts[q + 1] - cuts[q])
                    r = s.solve(sigma=sigma, k=6, config={"seed": 10 * t + i})
                    order = np.argsort(np.abs(w - sigma), kind="stable")
                    want, got = np.sort(w[order[:6]]), np.sort(r.eigenvalues)
                if not r.success or got.size != want.size or np.max(np.abs(got - want) / want) > EIG_RTOL:
                    errors.append((t, i, r.success, got.size, want.size))
        except Exception as e:  # reported below
            errors.append((t, repr(e)))
        finally:
            s.close()

    ths = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    assert not errors, errors


def _laplacian_2d(nx, ny):
    t1 = sp.diags([-np.ones(nx - 1), 2 * np.ones(nx), -np.ones(nx - 1)], [-1, 0, 1])
    t2 = sp.diags([-np.ones(ny - 1), 2 * np.ones(ny), -np.ones(ny - 1)], [-1, 0, 1])
    return (sp.kron(sp.identity(ny), t1) + sp.kron(t2, sp.identity(nx))).tocsr()


def test_smallest_and_largest_targets_standard_and_generalized():
    """Target modes smallest / largest (hsolve TargetMode::Smallest / Largest): the window closed by
    inertia search from a Ritz estimate of the spectrum's end, certified by counts; the k smallest
    ascending and the k largest descending, against dense eigenvalues."""
    import scipy.linalg as sla

    a = _laplacian_2d(30, 27)
    n = a.shape[0]
    rng = np.random.default_rng(11)
    off = sp.random(n, n, density=2.0 / n, random_state=3, format="csr")
    off = 0.05 * (off + off.T)
    bg = (off + sp.diags(1.0 + rng.uniform(0.0, 1.0, n) + abs(off).sum(axis=1).A1)).tocsr()
    bd = sp.diags(1.0 + rng.uniform(0.0, 1.0, n)).tocsr()
    for b in (None, bd, bg):
        w = sla.eigh(a.toarray(), None if b is None else b.toarray(), eigvals_only=True)
        r = hsolve.solve(a, b, k=7, mode="smallest")
        _check_pairs(r)
        np.testing.assert_allclose(r.eigenvalues, w[:7], rtol=EIG_RTOL)
        c = r.report["certificate"]
        assert c["passed"] and c["count_inertia"] >= 7
        r = hsolve.solve(a, b, k=5, mode="largest")
        _check_pairs(r)
        np.testing.assert_allclose(r.eigenvalues, w[::-1][:5], rtol=EIG_RTOL)
    # the Yee box's top end, against the exact spectrum
    box = yee.Box((8, 7, 6), (1.0, 0.9, 0.8))
    ay, by = yee.pencil(box, "generalized")
    wy = np.sort(yee_exact.exact_spectrum(box.cells, box.lengths))
    r = hsolve.solve(ay, by, k=6, mode="largest")
    _check_pairs(r)
    np.testing.assert_allclose(r.eigenvalues, wy[::-1][:6], rtol=EIG_RTOL)


@pytest.mark.parametrize("p", [1, 4, 8])
def test_krylov_basis_that_spans_the_whole_space(p):
    """A pencil so small that the Krylov basis spans the whole space: the next block is dependent on
    the basis to working precision (a block breakdown), the column-wise fallback leaves it with zero
    coupling instead of failing, and the Ritz pairs are exact. Also a block whose columns are nearly
    dependent (eigenvalues clustered to 1e-9): the conditioned CholQR2 path or its fallback must keep
    the basis orthonormal."""
    n = 48
    rng = np.random.default_rng(5)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    d = np.arange(1.0, n + 1.0)
    a = sp.csr_matrix(q @ np.diag(d) @ q.T)
    r = hsolve.solve(a, sigma=10.3, k=20, config={"block_size": p})
    _check_pairs(r)
    order = np.argsort(np.abs(d - 10.3), kind="stable")
    np.testing.assert_allclose(np.sort(r.eigenvalues), np.sort(d[order[:20]]), rtol=EIG_RTOL)
    d2 = np.concatenate([1.0 + 1e-9 * np.arange(8), np.linspace(3.0, 40.0, n - 8)])
    a2 = sp.csr_matrix(q @ np.diag(d2) @ q.T)
    r = hsolve.solve(a2, lower=0.5, upper=2.0, config={"block_size": p})
    _check_pairs(r)
    assert r.eigenvalues.size == 8
    np.testing.assert_allclose(r.eigenvalues, d2[:8], rtol=1e-9)
    x = r.eigenvectors
    assert np.abs(x.T @ x - np.eye(8)).max() < 1e-8
