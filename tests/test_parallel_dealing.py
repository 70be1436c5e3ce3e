"""CPU: multi-GPU dealing of slices and requests (hsolve_b200.parallel) - the cost-balanced deal, the
window plan by Sylvester counts, and the host gather of results over two and three gloo ranks, with
CPU stand-ins for the GPU count and solve (exact Yee spectra)."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

from hsolve_b200 import parallel
from oracle import yee_exact

ROOT = Path(__file__).resolve().parents[1]


def test_deal_is_balanced_complete_and_deterministic():
    rng = np.random.default_rng(0)
    costs = rng.uniform(1.0, 10.0, 37)
    for world in (1, 2, 3, 8):
        share = parallel.deal(costs, world)
        assert sorted(i for s in share for i in s) == list(range(37))
        loads = [costs[s].sum() for s in share]
        assert max(loads) - min(loads) <= costs.max() + 1e-12  # LPT: within one job of balance
        assert share == parallel.deal(list(costs), world)
    assert parallel.deal([], 4) == [[], [], [], []]


def test_plan_window_parts_count_the_whole_window():
    w = yee_exact.exact_spectrum((10, 9, 8))

    def count(s):
        return yee_exact.count_below(w, s)

    for parts in (1, 2, 3, 5):
        plan = parallel.plan_window(count, 40.0, 200.0, parts)
        assert plan[0].lower == 40.0 and plan[-1].upper == 200.0
        assert sum(p.count for p in plan) == count(200.0) - count(40.0)
        for p in plan:
            assert p.count == count(p.upper) - count(p.lower)
        if parts > 1:
            assert len(plan) >= 2


def test_plan_window_never_cuts_onto_a_multiple_eigenvalue():
    """Every eigenvalue of a spectrum of double eigenvalues: a goal count that falls between the two
    copies cannot be met, and the cut must go into a gap, well away from every eigenvalue."""
    base = np.sort(np.random.default_rng(3).uniform(40.0, 200.0, 25))
    w = np.repeat(base, 2)

    def count(s):
        return int(np.searchsorted(w, s, side="left"))

    for parts in (2, 3, 4, 7):
        plan = parallel.plan_window(count, 40.0, 200.0, parts)
        assert sum(p.count for p in plan) == w.size
        for p in plan[1:]:
            assert np.min(np.abs(w - p.lower)) > 1e-6 * 200.0, (parts, p)
            assert count(p.lower) % 2 == 0


def test_plan_window_skips_singular_counts():
    """A counter that reports None (a singular factorization) within 1e-9 of an eigenvalue, as the
    GPU count does when null-pivot detection fires: the plan must never take such a point, and a
    goal count between the copies of a double eigenvalue must not pull a cut onto it."""
    base = np.sort(np.random.default_rng(4).uniform(40.0, 200.0, 20))
    w = np.repeat(base, 2)
    seen = []

    def count(s):
        seen.append(s)
        if np.abs(w - s).min() < 1e-9 * 200.0:
            return None
        return int(np.searchsorted(w, s, side="left"))

    for parts in (2, 3, 5):
        plan = parallel.plan_window(count, 40.0, 200.0, parts)
        assert sum(p.count for p in plan) == w.size
        for p in plan[1:]:
            assert np.min(np.abs(w - p.lower)) > 1e-6 * 200.0, (parts, p)
    # a window end on an eigenvalue is moved until its count is regular
    plan = parallel.plan_window(count, float(base[0]), 200.0, 2)
    assert plan[0].lower != base[0] and abs(plan[0].lower - base[0]) < 1e-7 * 200.0
    assert sum(p.count for p in plan) == int(np.searchsorted(w, 200.0)) - int(np.searchsorted(w, plan[0].lower))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    from hsolve_b200 import parallel as par
    from oracle import yee_exact as ye

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = ye.exact_spectrum((10, 9, 8))
        solved = []

        def count(s):
            return ye.count_below(w, s)

        def solver(lo, hi):
            solved.append((lo, hi))
            lam = w[(w >= lo) & (w < hi)]
            return lam, np.ones((3, lam.size)), count(hi) - count(lo), True

        with par.Dealer() as d:
            lam, vec, rep = d.solve_interval(None, None, 40.0, 200.0, counter=count, solver=solver)
            reqs = [(np.zeros((n, n)), None, {}) for n in (5, 9, 7, 3)]
            res = d.solve_requests(reqs, solver=lambda a, b, t: (np.array([float(a.shape[0])]), True))
        out[rank] = (lam.tolist(), vec.shape, rep, solved, [(i, l.tolist(), ok) for i, l, ok in res])
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_dealer_gathers_every_part_once_over_gloo_ranks(world):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    w = yee_exact.exact_spectrum((10, 9, 8))
    want = w[(w >= 40.0) & (w < 200.0)]
    solved = [p for r in range(world) for p in res[r][3]]
    assert len(solved) == len(set(solved)) == len(res[0][2]["parts"])  # each part on exactly one rank
    assert all(len(res[r][3]) >= 1 for r in range(world))
    for r in range(world):
        lam, shape, rep, _, reqs = res[r]
        np.testing.assert_array_equal(lam, want)
        assert shape == (3, want.size)
        assert rep["passed"] and rep["count_found"] == rep["count_inertia"] == want.size and rep["ranks"] == world
        assert [i for i, _, _ in reqs] == [0, 1, 2, 3] and all(ok for _, _, ok in reqs)
        assert [v[0] for _, v, _ in reqs] == [5.0, 9.0, 7.0, 3.0]
