"""ORACLE (test infrastructure only): ctypes front end of oracle/_ref/libhsolve_ref.so, the parts of
the reference itself built from its sources by `make -C oracle ref` (its nested dissection,
include/hsolve/factor.hpp:631; its shifted residual and SpMM, include/hsolve/sparse.hpp:140-174).
Only tests/ import this module; available() is False where the library was not built.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np
import scipy.sparse as sp

SO = Path(__file__).resolve().parent / "_ref" / "libhsolve_ref.so"
_LIB = None


def available() -> bool:
    return SO.exists()


def _lib():
    global _LIB
    if _LIB is None:
        lib = ctypes.CDLL(str(SO))
        P, i64 = ctypes.c_void_p, ctypes.c_int64
        lib.ref_compute_ordering.argtypes = [i64, P, P, P, P, P, P, ctypes.c_uint64, ctypes.c_int, P, P]
        lib.ref_compute_ordering.restype = ctypes.c_int
        lib.ref_shifted_residual.argtypes = [i64, P, P, P, P, P, P, ctypes.c_double, P, P, P, i64, P]
        lib.ref_shifted_residual.restype = ctypes.c_int
        lib.ref_spmm.argtypes = [i64, P, P, P, P, P, i64]
        lib.ref_spmm.restype = ctypes.c_int
        _LIB = lib
    return _LIB


def _csr(m):
    m = sp.csr_matrix(m, dtype=np.float64)
    m.sum_duplicates()
    m.sort_indices()
    return (np.ascontiguousarray(m.indptr, dtype=np.int64), np.ascontiguousarray(m.indices, dtype=np.int32),
            np.ascontiguousarray(m.data, dtype=np.float64))


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def compute_ordering(a, b=None, seed: int = 2026, threads: int = 0):
    """(PERM_IN, top separator size) of the reference's nested dissection for the pencil (a, b)."""
    n = a.shape[0]
    ar = _csr(a)
    br = _csr(b) if b is not None else (None, None, None)
    perm = np.zeros(n, dtype=np.int32)
    top = ctypes.c_int64()
    rc = _lib().ref_compute_ordering(n, *map(_p, ar), *map(_p, br), seed, threads, _p(perm), ctypes.byref(top))
    if rc != 0:
        raise RuntimeError("reference compute_ordering failed")
    return perm, int(top.value)


def shifted_residual(a, b, sigma: float, x, y):
    """(R, omega): R = B X - (A Y - sigma B Y) and the componentwise backward errors (reference path)."""
    n = a.shape[0]
    x = np.asfortranarray(np.atleast_2d(x.T).T, dtype=np.float64)
    y = np.asfortranarray(np.atleast_2d(y.T).T, dtype=np.float64)
    p = x.shape[1]
    r = np.zeros((n, p), order="F")
    omega = np.zeros(p)
    ar = _csr(a)
    br = _csr(b) if b is not None else (None, None, None)
    rc = _lib().ref_shifted_residual(n, *map(_p, ar), *map(_p, br), float(sigma), _p(x), _p(y), _p(r), p, _p(omega))
    if rc != 0:
        raise RuntimeError("reference shifted_residual failed")
    return r, omega


def spmm(a, x):
    n = a.shape[0]
    x = np.asfortranarray(np.atleast_2d(x.T).T, dtype=np.float64)
    y = np.zeros_like(x, order="F")
    rc = _lib().ref_spmm(n, *map(_p, _csr(a)), _p(x), _p(y), x.shape[1])
    if rc != 0:
        raise RuntimeError("reference spmm failed")
    return y
