"""CPU: the native library loads, exports every entry point include/hsg.h declares, and its host-only
entry points (ordering, symbolic analysis) agree with the oracle."""
import re
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from hsolve_b200 import _native
from hsolve_b200.gen import yee
from oracle.ldlt import OracleLDLT

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        names |= set(re.findall(r"^HSG_API\s+[\w\s\*]+?\b(hsg_\w+)\s*\(", h.read_text(), flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    lib = _native.lib()
    names = declared_symbols()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
        assert name in _native.SIGNATURES, name


def test_status_strings_follow_reference_error_codes():
    lib = _native.lib()
    for status, name in _native.STATUS_NAMES.items():
        assert lib.hsg_status_string(status).decode() == name


def test_ordering_is_a_permutation_and_deterministic():
    a, _ = yee.pencil(yee.Box((9, 8, 7)))
    o1 = _native.compute_ordering(a)
    o2 = _native.compute_ordering(a)
    assert np.array_equal(np.sort(o1), np.arange(1, a.shape[0] + 1))
    assert np.array_equal(o1, o2)


def test_symbolic_matches_oracle_fill():
    """Fundamental supernodes on the same order: factor entries and flops equal the oracle's."""
    a, _ = yee.pencil(yee.Box((10, 9, 8)))
    n = a.shape[0]
    pos = _native.compute_ordering(a)
    perm = np.argsort(pos).astype(np.int32)
    st = _native.symbolic_stats(a, pos, amalgamate=False)
    o = OracleLDLT(a, order=perm)
    o.factorize(a + 50.0 * sp.identity(n))  # SPD: no pivoting, so no delays
    assert st["nnz_l"] == o.nnz_l
    assert abs(st["flops"] - o.flops) <= 1e-9 * o.flops
    st2 = _native.symbolic_stats(a, pos, amalgamate=True)
    assert st2["supernodes"] < st["supernodes"]
    assert st["flops"] <= st2["flops"] <= 1.2 * st["flops"]


def _brute_force_fill(a, pos):
    """Column counts of L for the 1-based pivot positions `pos` by explicit elimination of the graph:
    eliminating a vertex joins its not-yet-eliminated neighbours into a clique."""
    n = a.shape[0]
    order = np.argsort(pos)                      # pivot step -> vertex
    step = np.empty(n, dtype=np.int64)
    step[order] = np.arange(n)
    g = sp.csr_matrix(abs(a) + abs(a.T))
    adj = [set(g.indices[g.indptr[v]:g.indptr[v + 1]]) - {v} for v in range(n)]
    counts = np.zeros(n, dtype=np.int64)
    for v in order:
        later = [u for u in adj[v] if step[u] > step[v]]
        counts[step[v]] = len(later)
        for u in later:
            adj[u].update(w for w in later if w != u)
    return counts


@pytest.mark.parametrize("which", ["nd", "random", "natural"])
def test_symbolic_matches_brute_force_elimination(which):
    """nnz(L) and the RINFOG(1) flop count of the fundamental-supernode analysis equal an explicit
    elimination of the graph on the same order."""
    a, _ = yee.pencil(yee.Box((5, 4, 4)))
    n = a.shape[0]
    if which == "nd":
        pos = _native.compute_ordering(a)
    elif which == "random":
        pos = (np.random.default_rng(1).permutation(n) + 1).astype(np.int32)
    else:
        pos = np.arange(1, n + 1, dtype=np.int32)
    c = _brute_force_fill(a, pos)
    st = _native.symbolic_stats(a, pos, amalgamate=False)
    assert st["nnz_l"] == n + int(c.sum())
    flops = float(np.sum(c + c * (c + 1)))
    assert abs(st["flops"] - flops) <= 1e-12 * flops


def test_nested_dissection_beats_natural_order():
    a, _ = yee.pencil(yee.Box((12, 12, 12)))
    nd = _native.symbolic_stats(a, None)
    nat = _native.symbolic_stats(a, np.arange(1, a.shape[0] + 1, dtype=np.int32))
    assert nd["flops"] < 0.5 * nat["flops"]


def test_ordering_does_not_depend_on_thread_count():
    """The nested-dissection order is a function of the pattern and the seed only (hsolve's
    compute_ordering is thread-count independent, include/hsolve/factor.hpp:197-242)."""
    import os
    import subprocess
    import sys

    code = ("import sys, numpy as np; sys.path.insert(0, %r); import hsolve_b200 as hs; "
            "from hsolve_b200.gen import yee; a, _ = yee.pencil(yee.Box((18, 16, 14))); "
            "np.save(sys.argv[1], hs.compute_ordering(a))") % str(Path(__file__).resolve().parents[1])
    outs = []
    for threads in ("1", "3", "8"):
        path = Path(os.environ.get("TMPDIR", "/tmp")) / f"hsg_order_{os.getpid()}_{threads}.npy"
        env = dict(os.environ, HSOLVE_B200_ORDERING_THREADS=threads)
        subprocess.run([sys.executable, "-c", code, str(path)], check=True, env=env)
        outs.append(np.load(path))
        path.unlink()
    assert all(np.array_equal(outs[0], o) for o in outs[1:])
