"""Request-stream serving of certified eigensolves on one GPU.

    srv = Server(workers=3)
    fut = srv.submit(A, B, lower=lo, upper=hi)      # returns at once; fut.result() -> SolveResult
    ...
    srv.close(); print(srv.stats())                 # throughput and p50 / p99 latency

Requests of different sizes and shifts share the device: each runs in its own `Session` (its own
CUDA streams and factorization objects) on one of `workers` host threads, so the GPU interleaves the
latency-bound phases of several solves (continuous batching: a worker takes the next queued request
as soon as its last one finished). A request is admitted only when its device memory (from
the analysis of its pattern: factor storage of its factorization objects plus its Krylov basis)
fits the memory budget next to the requests already running; a pattern not seen before runs alone
the first time so that its footprint is known. Analyses and front plans are cached per sparsity
pattern inside the library, so a family of requests on one mesh (new Bloch wavevectors, new shifts,
new values) reuses one ordering, symbolic factorization and plan. Latency is measured from
submission (the request's arrival) to completion.

A pencil that many requests target can be registered: it then stays resident on the device, each
worker keeping its own session on it (created at the worker's first request and held until the
server closes), so its requests skip the upload, the analysis lookup and the norm estimates:

    h = srv.register(A, B)
    futs = [srv.submit(pencil=h, sigma=s, k=10) for s in shifts]
"""
from __future__ import annotations

import threading
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from .api import Session


@dataclass
class RequestRecord:
    n: int
    arrival: float
    start: float = 0.0
    end: float = 0.0
    device_mb: float = 0.0
    success: bool = False
    error: str = ""


@dataclass
class _Budget:
    total_mb: float
    used_mb: float = 0.0
    exclusive: bool = False
    active: int = 0
    cond: threading.Condition = field(default_factory=threading.Condition)


# device memory (MB) of a request, learned per (n, nnz(A), nnz(B), complex) the first time it runs;
# shared by every Server of the process, so reads and writes take _KNOWN_LOCK
_KNOWN_MB: dict[tuple, float] = {}
_KNOWN_LOCK = threading.Lock()


def _known_get(key):
    with _KNOWN_LOCK:
        return _KNOWN_MB.get(key)


def _known_set(key, mb: float) -> None:
    with _KNOWN_LOCK:
        _KNOWN_MB[key] = mb


def _free_device_mb(device: int) -> float:
    import torch

    free, _ = torch.cuda.mem_get_info(device)
    return free / 1e6


class Server:
    """Admits certified eigensolve requests by device memory and runs up to `workers` of them at
    once on `device` (see the module docstring)."""

    def __init__(self, workers: int = 3, memory_budget_gb: float | None = None, device: int = 0,
                 config: dict | None = None):
        if workers < 1:
            raise ValueError("workers must be >= 1")
        self.device = device
        self.config = dict(config or {})
        total = memory_budget_gb * 1e3 if memory_budget_gb is not None else 0.8 * _free_device_mb(device)
        self._budget = _Budget(total_mb=total)
        self._pool = ThreadPoolExecutor(max_workers=workers, thread_name_prefix="hsolve-serve")
        self._records: list[RequestRecord] = []
        self._lock = threading.Lock()
        self._pencils: dict[int, tuple] = {}  # registered pencils: handle -> (A, B, key)
        self._local = threading.local()      # per worker: handle -> its resident Session
        self._resident: list = []            # (Session, reserved MB) of every worker, closed with the server

    # ------------------------------------------------------------------------------ admission
    def _acquire(self, key, rec: RequestRecord) -> bool:
        """Blocks until the request fits; returns True when it runs alone (unknown footprint)."""
        b = self._budget
        with b.cond:
            known = _known_get(key)
            if known is None:
                b.cond.wait_for(lambda: b.active == 0)
                b.exclusive = True
                b.active += 1
                return True
            need = min(known, b.total_mb)
            b.cond.wait_for(lambda: not b.exclusive and b.used_mb + need <= b.total_mb)
            b.used_mb += need
            b.active += 1
            rec.device_mb = need
            return False

    def _release(self, alone: bool, rec: RequestRecord) -> None:
        b = self._budget
        with b.cond:
            if alone:
                b.exclusive = False
            else:
                b.used_mb -= rec.device_mb
            b.active -= 1
            b.cond.notify_all()

    def _reserve(self, mb: float) -> None:
        """Device memory held until the server closes (a worker's resident session)."""
        b = self._budget
        with b.cond:
            need = min(mb, b.total_mb)
            b.cond.wait_for(lambda: not b.exclusive and b.used_mb + need <= b.total_mb)
            b.used_mb += need

    # ------------------------------------------------------------------------------ requests
    def register(self, A, B=None) -> int:
        """Makes (A, B) a resident pencil and returns its handle for submit(pencil=...)."""
        key = (A.shape[0], getattr(A, "nnz", None), None if B is None else getattr(B, "nnz", None),
               bool(np.iscomplexobj(getattr(A, "data", np.zeros(0)))))
        with self._lock:
            h = len(self._pencils) + 1
            self._pencils[h] = (A, B, key)
        return h

    def submit(self, A=None, B=None, *, pencil: int | None = None, **target) -> Future:
        """Queue one solve (target keywords as in `hsolve_b200.solve`: sigma/k, lower/upper, tol,
        config) on the pencil (A, B), or on a registered pencil; the future's result is the
        SolveResult."""
        if pencil is not None:
            if pencil not in self._pencils:
                raise ValueError(f"unknown pencil handle {pencil}")
            A = self._pencils[pencil][0]
        elif A is None:
            raise ValueError("submit needs A or a registered pencil")
        rec = RequestRecord(n=A.shape[0], arrival=time.perf_counter())
        with self._lock:
            self._records.append(rec)
        if pencil is not None:
            return self._pool.submit(self._run_resident, pencil, target, rec)
        return self._pool.submit(self._run, A, B, target, rec)

    def _basis_mb(self, n: int) -> float:
        return 8.0 * 2 * n * 160 / 1e6

    def _run_resident(self, handle: int, target, rec: RequestRecord):
        A, B, key = self._pencils[handle]
        try:
            sessions = getattr(self._local, "sessions", None)
            if sessions is None:
                sessions = self._local.sessions = {}
            sess = sessions.get(handle)
            if sess is None:
                # the worker's own session on the pencil: its factor storage stays reserved
                if _known_get(key) is None:
                    alone = self._acquire(key, rec)
                    try:
                        sess = Session(A, B, device=self.device)
                        est = sess.estimate()
                        resident = 3.0 * est["device_mb"]
                        _known_set(key, resident + self._basis_mb(sess.n))
                    finally:
                        self._release(alone, rec)
                    self._reserve(resident)
                else:
                    resident = max(0.0, _known_get(key) - self._basis_mb(A.shape[0]))
                    self._reserve(resident)
                    sess = Session(A, B, device=self.device)
                with self._lock:
                    self._resident.append((sess, resident))
                sessions[handle] = sess
            # the request itself needs its Krylov basis next to the resident factors
            rec.device_mb = min(self._basis_mb(sess.n), self._budget.total_mb)
            b = self._budget
            with b.cond:
                b.cond.wait_for(lambda: not b.exclusive and b.used_mb + rec.device_mb <= b.total_mb)
                b.used_mb += rec.device_mb
                b.active += 1
            rec.start = time.perf_counter()
            try:
                cfg = dict(self.config)
                cfg.update(target.pop("config", None) or {})
                res = sess.solve(config=cfg, **target)
            finally:
                self._release(False, rec)
            rec.success = bool(res.success and res.report.get("certificate", {}).get("passed", True))
            return res
        except Exception as e:  # recorded, then re-raised through the future
            rec.error = f"{type(e).__name__}: {e}"
            raise
        finally:
            if rec.start == 0.0:
                rec.start = time.perf_counter()
            rec.end = time.perf_counter()

    def _run(self, A, B, target, rec: RequestRecord):
        key = (A.shape[0], getattr(A, "nnz", None), None if B is None else getattr(B, "nnz", None),
               bool(np.iscomplexobj(getattr(A, "data", np.zeros(0)))))
        alone = self._acquire(key, rec)
        rec.start = time.perf_counter()
        try:
            sess = Session(A, B, device=self.device)
            try:
                if alone:
                    est = sess.estimate()
                    # factor storage of up to three factorization objects plus the Krylov basis
                    basis_mb = self._basis_mb(sess.n)
                    rec.device_mb = 3.0 * est["device_mb"] + basis_mb
                    _known_set(key, rec.device_mb)
                cfg = dict(self.config)
                cfg.update(target.pop("config", None) or {})
                res = sess.solve(config=cfg, **target)
            finally:
                sess.close()
            rec.success = bool(res.success and res.report.get("certificate", {}).get("passed", True))
            return res
        except Exception as e:  # recorded, then re-raised through the future
            rec.error = f"{type(e).__name__}: {e}"
            raise
        finally:
            rec.end = time.perf_counter()
            self._release(alone, rec)

    def close(self, wait: bool = True) -> None:
        self._pool.shutdown(wait=wait)
        with self._lock:
            resident, self._resident = self._resident, []
        for sess, mb in resident:
            sess.close()
            with self._budget.cond:
                self._budget.used_mb -= min(mb, self._budget.total_mb)
                self._budget.cond.notify_all()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------------------ metrics
    def stats(self) -> dict:
        """Throughput of certified solves and latency percentiles of the completed requests."""
        with self._lock:
            done = [r for r in self._records if r.end > 0]
        if not done:
            return {"requests": 0}
        lat = np.array([r.end - r.arrival for r in done])
        service = np.array([r.end - r.start for r in done])
        span = max(r.end for r in done) - min(r.arrival for r in done)
        ok = sum(r.success for r in done)
        return {"requests": len(done), "certified": ok, "failed": [r.error for r in done if r.error],
                "solves_per_s": ok / span if span > 0 else 0.0, "makespan_s": span,
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "service_mean_s": float(service.mean())}
