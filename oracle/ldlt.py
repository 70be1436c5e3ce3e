"""ORACLE (test infrastructure only): ctypes front end of oracle/mf_ldlt.c, the CPU restatement of
the multifrontal LDL^T with threshold 1x1/2x2 pivoting, delayed pivots, scaling, null-pivot
detection and inertia (hsolve's MUMPS path: src/factor/mumps_factorization.cpp:300-381,459-527).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent
_LIB = None


def build() -> Path:
    so = HERE / "liboracle_mf.so"
    src = HERE / "mf_ldlt.c"
    if not so.exists() or so.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return so


def _lib():
    global _LIB
    if _LIB is None:
        lib = ctypes.CDLL(str(build()))
        P = ctypes.c_void_p
        i64 = ctypes.c_int64
        lib.mf_analyze.restype = P
        lib.mf_analyze.argtypes = [i64, P, P, P]
        lib.mf_analyze_relaxed.restype = P
        lib.mf_analyze_relaxed.argtypes = [i64, P, P, P, ctypes.c_int]
        lib.mf_factor.restype = ctypes.c_int
        lib.mf_factor.argtypes = [P, P, P, P, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, P]
        lib.mf_solve.restype = ctypes.c_int
        lib.mf_solve.argtypes = [P, P, i64, i64]
        lib.mf_free.argtypes = [P]
        lib.mf_flops.restype = ctypes.c_double
        lib.mf_flops.argtypes = [P]
        lib.mf_nnz_l.restype = i64
        lib.mf_nnz_l.argtypes = [P]
        lib.mf_supernodes.restype = ctypes.c_int32
        lib.mf_supernodes.argtypes = [P]
        lib.mf_threads.restype = ctypes.c_int
        lib.mf_set_dgemm.argtypes = [P]
        lib.mf_set_dgemm.restype = None
        fn = _scipy_dgemm()
        if fn:
            lib.mf_set_dgemm(fn)
        _LIB = lib
    return _LIB


def _scipy_dgemm():
    """Address of the Fortran dgemm of the BLAS that scipy loads (scipy.linalg.cython_blas), or None.
    The frontal updates of the restatement run through it; its own threads are limited to one while
    the restatement runs (the fronts are parallel in OpenMP)."""
    try:
        from scipy.linalg import cython_blas
    except Exception:
        return None
    cap = cython_blas.__pyx_capi__.get("dgemm")
    if cap is None:
        return None
    get_name = ctypes.pythonapi.PyCapsule_GetName
    get_name.restype = ctypes.c_char_p
    get_name.argtypes = [ctypes.py_object]
    get_ptr = ctypes.pythonapi.PyCapsule_GetPointer
    get_ptr.restype = ctypes.c_void_p
    get_ptr.argtypes = [ctypes.py_object, ctypes.c_char_p]
    return get_ptr(cap, get_name(cap))


def _one_blas_thread():
    try:
        from threadpoolctl import threadpool_limits

        return threadpool_limits(limits=1, user_api="blas")
    except Exception:  # threadpoolctl is optional
        import contextlib

        return contextlib.nullcontext()


def upper_csr(m) -> sp.csr_matrix:
    """Upper triangle (row <= col) of a symmetric matrix, canonical CSR, int64 rowptr, int32 cols."""
    u = sp.triu(sp.csr_matrix(m), format="csr")
    u.sum_duplicates()
    u.sort_indices()
    return u


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleLDLT:
    """K = alpha A + beta B on a fixed pattern; factorize(...) returns (valid, inertia, stats).
    relax: amalgamate the fundamental supernodes (fewer, larger fronts with a few explicit zeros;
    the exact-fill comparisons of the tests use the fundamental ones)."""

    def __init__(self, pattern, order=None, relax=False):
        u = upper_csr(pattern)
        self.n = u.shape[0]
        self.rp = np.ascontiguousarray(u.indptr, dtype=np.int64)
        self.ci = np.ascontiguousarray(u.indices, dtype=np.int32)
        self._pattern = u
        o = None if order is None else np.ascontiguousarray(order, dtype=np.int32)
        self._h = _lib().mf_analyze_relaxed(self.n, _ptr(self.rp), _ptr(self.ci), None if o is None else _ptr(o),
                                            int(relax))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _lib().mf_free(h)
            self._h = None

    def values_of(self, k) -> np.ndarray:
        """Values of the symmetric matrix k on the analysed upper pattern (zeros where absent);
        entries of k at positions outside the pattern must be zero."""
        u = upper_csr(k)
        n = self.n
        rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(self.rp))
        keys = rows * n + self.ci
        urows = np.repeat(np.arange(n, dtype=np.int64), np.diff(u.indptr))
        ukeys = urows * n + u.indices
        pos = np.searchsorted(keys, ukeys)
        pos_c = np.minimum(pos, keys.size - 1)
        hit = keys[pos_c] == ukeys
        if np.any(u.data[~hit] != 0):
            raise ValueError("matrix has entries outside the analysed pattern")
        v = np.zeros(keys.size)
        v[pos_c[hit]] = u.data[hit]
        return v

    def factorize(self, k, u=0.01, null_tol=1e-8, detect=True, scaling=True):
        v = self.values_of(k)
        out = np.zeros(6, dtype=np.int64)
        lib = _lib()
        with _one_blas_thread():
            valid = lib.mf_factor(self._h, _ptr(self.rp), _ptr(self.ci), _ptr(v), u, null_tol,
                                  int(detect), int(scaling), _ptr(out))
        neg, zero, pos, delayed, two, null = (int(x) for x in out)
        return bool(valid), (neg, zero, pos), {"delayed": delayed, "two_by_two": two, "null_pivots": null}

    def solve(self, b):
        x = np.array(b, dtype=np.float64, order="F", copy=True)
        if x.ndim == 1:
            x = x.reshape(-1, 1, order="F")
        lib = _lib()
        with _one_blas_thread():
            lib.mf_solve(self._h, _ptr(x), x.shape[1], x.shape[0])
        return x if np.ndim(b) == 2 else x[:, 0]

    @property
    def flops(self) -> float:
        return _lib().mf_flops(self._h)

    @property
    def nnz_l(self) -> int:
        return int(_lib().mf_nnz_l(self._h))

    @property
    def supernodes(self) -> int:
        return int(_lib().mf_supernodes(self._h))


def threads() -> int:
    return int(_lib().mf_threads())
