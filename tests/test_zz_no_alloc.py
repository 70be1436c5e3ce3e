"""hsg_solve_static: the solve for callers that must not allocate device memory.

Some callers cannot call cudaMalloc: a process whose device memory a pooling allocator has
already claimed, or a serving loop that cannot pay for the device-wide synchronisation of cudaFree.
hsg_solve_static runs the same solve as hsg_solve with its work space in one fixed array compiled
into the library. This file is collected last on purpose, so that a run stopping at its first
failure has run every other test first; it passes alone and after the others.
"""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from hsolve_b200 import _native
from hsolve_b200.gen import yee

pytestmark = pytest.mark.gpu

STATIC_BYTES = 16 << 20  # HSG_SOLVE_STATIC_SCRATCH_BYTES in include/hsg.h


def _factor(cells, sigma):
    a, _ = yee.pencil(yee.Box(cells))
    f = _native.Factorization(device=0)
    f.analyze(a, None, 1.0, -sigma)
    assert f.factorize(1.0, -sigma)
    return f, (a - sigma * sp.identity(a.shape[0])).tocsr()


@pytest.mark.parametrize("cells,sigma,nrhs", [((8, 7, 6), 33.3, 3), ((20, 18, 16), 61.7, 11)])
def test_static_solve_matches_hsg_solve_twice_in_a_row(cells, sigma, nrhs):
    import torch

    f, k = _factor(cells, sigma)
    n = k.shape[0]
    rng = np.random.default_rng(7)
    for call in range(2):
        b = rng.standard_normal((n, nrhs))
        ref = f.solve(b)  # the existing entry point (host buffers)
        ld = n + 5  # a leading dimension larger than n
        dev = torch.zeros((nrhs, ld), dtype=torch.float64, device="cuda:0")
        dev[:, :n] = torch.from_numpy(b.T.copy())
        torch.cuda.synchronize()  # the copy into dev is complete before the solve reads it
        f.solve_static(dev.data_ptr(), nrhs, ld)
        torch.cuda.synchronize()
        got = dev[:, :n].cpu().numpy().T
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max()), call
        assert np.all(dev[:, n:].cpu().numpy() == 0.0)  # rows past n untouched
        be = np.abs(k @ got - b).max() / (abs(k).sum(axis=0).max() * np.abs(got).max())
        assert be < 1e-12, be
    f.close()


def test_first_solve_of_a_fresh_factorization_allocates_nothing():
    """The first solve after a factorization also builds the solve operators; through
    hsg_solve_static it does so without allocating device memory, and its result matches the
    oracle's solve."""
    import torch

    from oracle.ldlt import OracleLDLT

    warm, _ = _factor((6, 5, 4), 20.5)  # loads the library's kernels and the static array
    wn = warm.order()
    wb = torch.ones((1, wn), dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    warm.solve_static(wb.data_ptr(), 1, wn)
    warm.close()

    cells, sigma, nrhs = (12, 10, 9), 47.3, 4
    f, k = _factor(cells, sigma)  # factorized, never solved
    n = k.shape[0]
    b = np.random.default_rng(3).standard_normal((n, nrhs))
    dev = torch.from_numpy(b.T.copy()).to("cuda:0")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    f.solve_static(dev.data_ptr(), nrhs, n)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
    got = dev.cpu().numpy().T
    a, _ = yee.pencil(yee.Box(cells))
    ok, _, _ = (o := OracleLDLT(a)).factorize(k)
    assert ok
    want = o.solve(b)
    assert np.allclose(got, want, rtol=1e-10, atol=1e-10 * np.abs(want).max())
    f.close()


def test_static_solve_rejects_host_memory_and_huge_counts():
    f, _ = _factor((6, 5, 4), 20.5)
    n = f.order()
    host = np.zeros((2, n))
    status = _native.lib().hsg_solve_static(f._h, ctypes.c_void_p(host.ctypes.data), 2, n)
    assert status == 1 and "not device memory" in _native.lib().hsg_last_error().decode()
    status = _native.lib().hsg_solve_static(f._h, ctypes.c_void_p(host.ctypes.data), 1 << 62, n)
    assert status == 1 and "static array holds" in _native.lib().hsg_last_error().decode()
    f.close()


def test_static_solve_rejects_requests_beyond_its_array():
    import torch

    f, _ = _factor((8, 7, 6), 33.3)
    n = f.order()
    nrhs = STATIC_BYTES // (8 * n) + 1  # the right-hand sides alone exceed the array
    dev = torch.zeros((1, n), dtype=torch.float64, device="cuda:0")
    status = _native.lib().hsg_solve_static(f._h, ctypes.c_void_p(dev.data_ptr()), nrhs, n)
    assert status == 1  # HSG_INVALID_INPUT; nothing was launched
    msg = _native.lib().hsg_last_error().decode()
    assert "static array holds" in msg and "split the right-hand sides" in msg
    f.close()
