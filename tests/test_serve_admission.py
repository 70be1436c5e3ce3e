"""CPU: admission and accounting of the request server (hsolve_b200.serve.Server), with a stand-in
session that sleeps instead of solving. What is checked is the server's own logic: a pattern seen
for the first time runs alone; known patterns run concurrently as far as `workers` and the device
memory budget allow; failures are recorded and re-raised through the future; stats() reports
counts and latency percentiles.
"""
import threading
import time
from types import SimpleNamespace

import numpy as np
import pytest
import scipy.sparse as sp

from hsolve_b200 import serve


class _Tracker:
    def __init__(self):
        self.lock = threading.Lock()
        self.active = 0
        self.max_active = 0
        self.log = []  # (event, n, active after the event)

    def enter(self, n):
        with self.lock:
            self.active += 1
            self.max_active = max(self.max_active, self.active)
            self.log.append(("start", n, self.active))

    def leave(self, n):
        with self.lock:
            self.active -= 1
            self.log.append(("end", n, self.active))


def _fake_session_class(tracker, device_mb, fail_n=None, dt=0.05):
    class FakeSession:
        def __init__(self, A, B=None, device=0):
            self.n = A.shape[0]

        def estimate(self):
            return {"device_mb": device_mb(self.n)}

        def solve(self, config=None, **target):
            tracker.enter(self.n)
            try:
                time.sleep(dt)
                if fail_n is not None and self.n == fail_n:
                    raise RuntimeError("stand-in failure")
                return SimpleNamespace(success=True, report={"certificate": {"passed": True}})
            finally:
                tracker.leave(self.n)

        def close(self):
            pass

    return FakeSession


@pytest.fixture(autouse=True)
def _fresh_cache(monkeypatch):
    monkeypatch.setattr(serve, "_KNOWN_MB", {})


def _mat(n):
    return sp.identity(n, format="csr")


def test_new_pattern_runs_alone_then_known_ones_overlap(monkeypatch):
    tr = _Tracker()
    monkeypatch.setattr(serve, "Session", _fake_session_class(tr, lambda n: 1.0))
    srv = serve.Server(workers=3, memory_budget_gb=100.0)
    first = [srv.submit(_mat(50), lower=0.0, upper=1.0) for _ in range(4)]
    for f in first:
        assert f.result().success
    srv.close()
    # the first request of the pattern ran with nothing else active
    assert tr.log[0] == ("start", 50, 1) and tr.log[1] == ("end", 50, 0)
    # the other three (known footprint, budget ample) overlapped up to the worker count
    assert tr.max_active == 3
    st = srv.stats()
    assert st["requests"] == 4 and st["certified"] == 4 and not st["failed"]
    assert st["latency_p99_s"] >= st["latency_p50_s"] > 0 and st["solves_per_s"] > 0


def test_memory_budget_limits_concurrency(monkeypatch):
    tr = _Tracker()
    # each request of this pattern needs 605 MB (3 factorization objects x 200 MB + 5 MB of Krylov
    # basis), so only one fits in a 1 GB budget at a time
    monkeypatch.setattr(serve, "Session", _fake_session_class(tr, lambda n: 200.0))
    srv = serve.Server(workers=4, memory_budget_gb=1.0)
    futs = [srv.submit(_mat(2000), sigma=1.0, k=2) for _ in range(5)]
    for f in futs:
        f.result()
    srv.close()
    assert tr.max_active == 1
    need = serve._KNOWN_MB[(2000, 2000, None, False)]
    assert 600.0 < need < 1000.0


def test_request_above_budget_still_runs(monkeypatch):
    tr = _Tracker()
    monkeypatch.setattr(serve, "Session", _fake_session_class(tr, lambda n: 10_000.0))
    srv = serve.Server(workers=2, memory_budget_gb=1.0)
    futs = [srv.submit(_mat(30), sigma=1.0, k=1) for _ in range(3)]
    assert all(f.result().success for f in futs)
    srv.close()
    assert tr.max_active == 1


def test_failure_is_recorded_and_reraised(monkeypatch):
    tr = _Tracker()
    monkeypatch.setattr(serve, "Session", _fake_session_class(tr, lambda n: 1.0, fail_n=77))
    srv = serve.Server(workers=2, memory_budget_gb=10.0)
    ok = srv.submit(_mat(40), sigma=1.0, k=1)
    bad = srv.submit(_mat(77), sigma=1.0, k=1)
    assert ok.result().success
    with pytest.raises(RuntimeError, match="stand-in failure"):
        bad.result()
    srv.close()
    st = srv.stats()
    assert st["requests"] == 2 and st["certified"] == 1
    assert len(st["failed"]) == 1 and "stand-in failure" in st["failed"][0]
    # the failed request released its admission: the budget is free again
    assert srv._budget.used_mb == 0.0 and srv._budget.active == 0 and not srv._budget.exclusive


def test_workers_must_be_positive():
    with pytest.raises(ValueError):
        serve.Server(workers=0, memory_budget_gb=1.0)


def test_mixed_sizes_keys_are_separate(monkeypatch):
    tr = _Tracker()
    monkeypatch.setattr(serve, "Session", _fake_session_class(tr, lambda n: 1.0, dt=0.02))
    srv = serve.Server(workers=3, memory_budget_gb=10.0)
    sizes = [20, 30, 20, 30, 20, 30]
    futs = [srv.submit(_mat(n), sigma=1.0, k=1) for n in sizes]
    for f in futs:
        f.result()
    srv.close()
    assert set(k[0] for k in serve._KNOWN_MB) == {20, 30}
    # each size's first request started with nothing else running
    firsts = {}
    for ev, n, active in tr.log:
        if ev == "start" and n not in firsts:
            firsts[n] = active
    assert firsts == {20: 1, 30: 1}
    assert np.isfinite(srv.stats()["makespan_s"])


def test_registered_pencil_keeps_one_session_per_worker(monkeypatch):
    """A registered pencil: each worker builds its own session once and reuses it for every later
    request; the sessions' memory stays reserved until close() releases it."""
    tr = _Tracker()
    made = []
    base = _fake_session_class(tr, lambda n: 2.0)

    class Counting(base):
        def __init__(self, *a, **k):
            super().__init__(*a, **k)
            made.append(self)

    monkeypatch.setattr(serve, "Session", Counting)
    srv = serve.Server(workers=3, memory_budget_gb=100.0)
    h = srv.register(_mat(40))
    futs = [srv.submit(pencil=h, sigma=0.5, k=2) for _ in range(12)]
    assert all(f.result().success for f in futs)
    assert 1 <= len(made) <= 3
    assert tr.max_active <= 3
    assert srv._budget.used_mb > 0  # resident sessions hold their factor storage
    srv.close()
    assert abs(srv._budget.used_mb) < 1e-9
    st = srv.stats()
    assert st["requests"] == 12 and st["certified"] == 12
    with pytest.raises(ValueError):
        srv.submit(pencil=99, sigma=0.0, k=1)
