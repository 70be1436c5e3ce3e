"""Multi-GPU dealing of independent work: spectrum slices of one interval, or serving requests.

One process per GPU (torch.distributed, NCCL on GPUs, gloo on CPU). The path shards by independent
problems, with no data-path collective: slices of one interval are independent shifts after one
shared analysis, and requests are independent pencils (the reference's helper scheme,
include/hsolve/parallel.hpp:3-17, with slices as the unit, src/driver/definite.cpp:1193). Work is
dealt by predicted cost (longest first to the least-loaded rank); every rank solves its share with
its own Session, and the host gathers eigenpairs and Sylvester counts (integers) at the end.

    with Dealer() as d:                                  # inside a torchrun launch
        res = d.solve_interval(A, B, lower, upper)       # every rank returns the whole result

Cost model of a slice with c eigenvalues: one factorization plus c / p block solves of a Krylov
basis of about 2c + 16 vectors, i.e. proportional to (1 + c / 8); of a request: its factorization
flops estimate (the symbolic analysis), else n^1.5.
"""
from __future__ import annotations

import heapq
from dataclasses import dataclass

import numpy as np


def deal(costs, world: int) -> list[list[int]]:
    """Indices of `costs` per rank: longest processing time first, each to the least-loaded rank
    (ties to the lowest rank), so the result is deterministic on every rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    share: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        share[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    for s in share:
        s.sort()
    return share


def slice_cost(count: int) -> float:
    return 1.0 + count / 8.0


@dataclass
class WindowPart:
    lower: float
    upper: float
    count: int


def _count_near(count_below, s: float, step: float, tries: int = 4):
    """(point, count) at s, or at s + step, s - 2 step, s + 3 step, ... when the count at s is None
    (a singular factorization: s lies on an eigenvalue to working precision); (s, None) if every
    try was singular."""
    for t in range(tries + 1):
        x = s + (t if t % 2 else -t) * step if t else s
        n = count_below(x)
        if n is not None:
            return x, n
    return s, None


def _bisect(count_below, lo: float, hi: float, goal: int, steps: int):
    """First bisection point s of (lo, hi) with count_below(s) == goal: (s, None), or (None, (a, b,
    n_a, n_b)) with the final bracket when no point of the search had that count."""
    a, b = lo, hi
    na = nb = None
    for _ in range(steps):
        mid, nm = _count_near(count_below, 0.5 * (a + b), 1e-3 * (b - a))
        if nm is None:
            break
        if nm == goal:
            return mid, None
        if nm < goal:
            a, na = mid, nm
        else:
            b, nb = mid, nm
    return None, (a, b, na, nb)


def plan_window(count_below, lower: float, upper: float, parts: int, max_bisect: int = 40) -> list[WindowPart]:
    """Sub-windows of [lower, upper) holding about equal numbers of eigenvalues: `count_below(s)`
    is the Sylvester count nu_-(A - s B) of an FP64 factorization, or None when that factorization
    is singular (s on an eigenvalue to working precision; such a point is never used). Cut points
    are placed by bisection on the count; every part carries its certified count. A multiple
    eigenvalue that straddles a goal count cannot be split: the search then takes the count just
    below it (or, if that adds nothing, just above it) and cuts at the first bisection point of the
    gap next to it, so that no cut converges onto an eigenvalue. A singular window end is moved by
    a few multiples of 1e-9 of the window width until its factorization is regular."""
    width = upper - lower
    lower, n_lo = _count_near(count_below, lower, -1e-9 * width)
    upper, n_hi = _count_near(count_below, upper, 1e-9 * width)
    if n_lo is None or n_hi is None:
        raise ValueError("plan_window: the window ends stay singular after moves")
    total = n_hi - n_lo
    parts = max(1, min(parts, total)) if total > 0 else 1
    cuts, below = [lower], [n_lo]
    for q in range(1, parts):
        goal = n_lo + round(q * total / parts)
        if goal <= below[-1] or goal >= n_hi:
            continue
        s, bracket = _bisect(count_below, cuts[-1], upper, goal, max_bisect)
        got = goal
        if s is None:
            a, b, na, nb = bracket
            if na is not None and na > below[-1]:
                got = na
                s, _ = _bisect(count_below, cuts[-1], a, na, max_bisect)
            elif nb is not None and nb < n_hi:
                got = nb
                s, _ = _bisect(count_below, b, upper, nb, max_bisect)
        if s is not None and got > below[-1]:
            cuts.append(s)
            below.append(got)
    cuts.append(upper)
    below.append(n_hi)
    return [WindowPart(cuts[i], cuts[i + 1], below[i + 1] - below[i]) for i in range(len(cuts) - 1)]


def gather_results(dist, local: list[tuple[int, np.ndarray, np.ndarray, int, bool]]):
    """All ranks' (part index, eigenvalues, eigenvectors, counted, certified) on every rank, in part
    order (all_gather_object: the host exchange of the result; no collective on the data path)."""
    world = dist.get_world_size()
    everything = [None] * world
    dist.all_gather_object(everything, local)
    merged = [item for share in everything for item in share]
    merged.sort(key=lambda t: t[0])
    return merged


class Dealer:
    """Slices of one interval, or a list of requests, dealt over the ranks of the current process
    group (a single process acts as one rank)."""

    def __init__(self, device: int | None = None):
        import torch.distributed as dist

        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.rank = self.dist.get_rank() if self.dist else 0
        self.world = self.dist.get_world_size() if self.dist else 1
        self.device = device if device is not None else 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def solve_interval(self, A, B, lower: float, upper: float, config: dict | None = None, counter=None,
                       solver=None, parts: int | None = None):
        """All eigenpairs in [lower, upper): the window is cut into `parts` parts (default: one per
        rank) of about equal count, parts are dealt by cost, each rank certifies its parts, the host
        gathers. `counter(s)` / `solver(lower, upper)` default to the GPU library (tests pass CPU
        stand-ins)."""
        if counter is None or solver is None:
            from . import _native
            from .api import Session

            if counter is None:
                f = _native.Factorization(device=self.device)
                f.analyze(A, B, 1.0, -0.5 * (lower + upper))

                def counter(s, _f=f):
                    r = _f.count(1.0, -s)
                    return r.neg if r.valid else None

            if solver is None:
                sess = Session(A, B, device=self.device)

                def solver(lo, hi, _s=sess):
                    r = _s.solve(lower=lo, upper=hi, config=config or {})
                    c = r.report["certificate"]
                    return r.eigenvalues, r.eigenvectors, int(c["count_inertia"]), bool(r.success)

        parts = plan_window(counter, lower, upper, parts or self.world)
        share = deal([slice_cost(p.count) for p in parts], self.world)[self.rank]
        local = []
        for i in share:
            lam, vec, counted, ok = solver(parts[i].lower, parts[i].upper)
            local.append((i, np.asarray(lam), np.asarray(vec), counted, ok and counted == parts[i].count))
        merged = gather_results(self.dist, local) if self.dist else sorted(local, key=lambda t: t[0])
        lam = np.concatenate([m[1] for m in merged]) if merged else np.zeros(0)
        vec = np.hstack([m[2] for m in merged]) if merged else None
        total = sum(p.count for p in parts)
        certified = all(m[4] for m in merged) and lam.size == total
        return lam, vec, {"parts": [(p.lower, p.upper, p.count) for p in parts], "count_inertia": total,
                          "count_found": int(lam.size), "passed": certified, "ranks": self.world}

    def solve_requests(self, requests, costs=None, solver=None):
        """Every request (A, B, target dict) solved by one rank, dealt by predicted cost; returns the
        list of (index, result summary) of all requests on every rank."""
        if costs is None:
            costs = [float(a.shape[0]) ** 1.5 for a, _, _ in requests]
        share = deal(costs, self.world)[self.rank]
        if solver is None:
            from .api import solve as _solve

            def solver(a, b, target):
                r = _solve(a, b, config={"device": self.device}, **target)
                return r.eigenvalues, bool(r.success)

        local = []
        for i in share:
            a, b, t = requests[i]
            lam, ok = solver(a, b, t)
            local.append((i, np.asarray(lam), None, 0, ok))
        merged = gather_results(self.dist, local) if self.dist else sorted(local, key=lambda t: t[0])
        return [(m[0], m[1], m[4]) for m in merged]
