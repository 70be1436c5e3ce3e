"""ctypes binding of the C ABI (include/hsg.h) in hsolve_b200/lib/libhsolve_b200.so.

`Factorization` mirrors hs::SparseFactorization<double> (hsolve include/hsolve/factor.hpp:341-443):
analyze / estimate / factorize / count / solve / inertia / release_factors /
set_null_pivot_detection / pivot_order / order, with hsolve's error classes raised from the status
codes. The library is required: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libhsolve_b200.so"

_lib = None


class _Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("null_pivot_tol", ctypes.c_double),
                ("single_null_pivot_tol", ctypes.c_double), ("pivot_threshold", ctypes.c_double),
                ("device", ctypes.c_int32), ("ordering_seed", ctypes.c_uint64), ("scaling", ctypes.c_int32)]


class _Inertia(ctypes.Structure):
    _fields_ = [("neg", ctypes.c_int64), ("zero", ctypes.c_int64), ("pos", ctypes.c_int64),
                ("valid", ctypes.c_int32), ("null_pivots", ctypes.c_int64), ("delayed_pivots", ctypes.c_int64),
                ("two_by_two", ctypes.c_int64), ("replans", ctypes.c_int32)]


class _Estimate(ctypes.Structure):
    _fields_ = [("factor_entries", ctypes.c_int64), ("nnz_l", ctypes.c_int64), ("flops", ctypes.c_double),
                ("device_mb", ctypes.c_double), ("supernodes", ctypes.c_int32), ("levels", ctypes.c_int32),
                ("max_front", ctypes.c_int32), ("ordering_s", ctypes.c_double), ("analyze_s", ctypes.c_double)]


# hs::Error::Code names in status order (status = code + 1), include/hsolve/error.hpp:16-26
STATUS_NAMES = {0: "ok", 1: "invalid_input", 2: "io", 3: "not_hermitian", 4: "unsupported",
                5: "factorization_failed", 6: "singular", 7: "out_of_memory_budget", 8: "not_converged",
                9: "internal"}

# C declarations of include/hsg.h: name -> (restype, argtypes)
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I32 = ctypes.c_int32
_D = ctypes.c_double
SIGNATURES = {
    "hsg_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "hsg_last_error": (ctypes.c_char_p, []),
    "hsg_kernel_launches": (ctypes.c_int64, []),
    "hsg_fp64_peak_probe": (ctypes.c_int, [_I32, _P]),
    "hsg_default_options": (None, [_P]),
    "hsg_create": (ctypes.c_int, [_P, _P]),
    "hsg_destroy": (ctypes.c_int, [_P]),
    "hsg_analyze": (ctypes.c_int, [_P, _I64, _P, _P, _P, _P, _P, _P, _D, _D, _P]),
    "hsg_estimate": (ctypes.c_int, [_P, _P]),
    "hsg_factorize": (ctypes.c_int, [_P, _D, _D, _P]),
    "hsg_count": (ctypes.c_int, [_P, _D, _D, _I32, _P]),
    "hsg_solve": (ctypes.c_int, [_P, _P, _I64, _I64, _I32]),
    "hsg_solve_static": (ctypes.c_int, [_P, _P, _I64, _I64]),
    "hsg_inertia": (ctypes.c_int, [_P, _P]),
    "hsg_release": (ctypes.c_int, [_P, _P]),
    "hsg_set_null_pivot_detection": (ctypes.c_int, [_P, _I32]),
    "hsg_pivot_order": (ctypes.c_int, [_P, _P]),
    "hsg_order": (_I64, [_P]),
    "hsg_clear_analysis_cache": (ctypes.c_int, []),
    "hsg_spmm": (ctypes.c_int, [_I64, _P, _P, _P, _P, _I64, _P, _I64, _I64, _D, _D]),
    "hsg_shifted_residual": (ctypes.c_int, [_I64, _P, _P, _P, _P, _P, _P, _D, _P, _I64, _P, _I64, _P, _I64, _I64,
                                            _P]),
    "hsg_compute_ordering": (ctypes.c_int, [_I64, _P, _P, ctypes.c_uint64, _P]),
    "hsg_symbolic_stats": (ctypes.c_int, [_I64, _P, _P, _P, _I32, _P]),
    "hsg_csr_inspect": (ctypes.c_int, [_I64, _P, _P, _P, _P, _P, _P, _P]),
}


def lib():
    """The loaded native library (raises if it was not built: no fallback exists)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"native library missing: {LIB_PATH} (run python -m hsolve_b200.build)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != 0:
        from . import errors

        msg = lib().hsg_last_error().decode(errors="replace")
        raise errors.from_code(STATUS_NAMES.get(status, "internal"), msg)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def upper_csr(m):
    """Upper triangle (row <= col) of a symmetric matrix as (rowptr int64, col int32, val float64)."""
    import scipy.sparse as sp

    u = sp.triu(sp.csr_matrix(m), format="csr")
    u.sum_duplicates()
    u.sort_indices()
    return (np.ascontiguousarray(u.indptr, dtype=np.int64), np.ascontiguousarray(u.indices, dtype=np.int32),
            np.ascontiguousarray(u.data, dtype=np.float64))


@dataclass
class Inertia:
    """hs::Inertia (factor.hpp:295-300) with the pivot statistics of the factorization."""
    neg: int
    zero: int
    pos: int
    valid: bool
    null_pivots: int = 0
    delayed_pivots: int = 0
    two_by_two: int = 0
    replans: int = 0


def _inertia(c: _Inertia) -> Inertia:
    return Inertia(int(c.neg), int(c.zero), int(c.pos), bool(c.valid), int(c.null_pivots), int(c.delayed_pivots),
                   int(c.two_by_two), int(c.replans))


def default_options() -> dict:
    o = _Options()
    lib().hsg_default_options(ctypes.byref(o))
    return {f: getattr(o, f) for f, _ in _Options._fields_}


class Factorization:
    """GPU sparse LDL^T of K = alpha A + beta B on a fixed pattern (SparseFactorization<double>)."""

    def __init__(self, **options):
        o = _Options()
        lib().hsg_default_options(ctypes.byref(o))
        for k, v in options.items():
            if not hasattr(o, k):
                raise TypeError(f"unknown option {k!r}")
            setattr(o, k, v)
        h = ctypes.c_void_p()
        check(lib().hsg_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self._keep = []

    def close(self):
        if getattr(self, "_h", None):
            lib().hsg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def analyze(self, A, B=None, alpha=1.0, beta=0.0, pivot_order=None):
        arp, aci, av = upper_csr(A)
        n = A.shape[0]
        if B is not None:
            brp, bci, bv = upper_csr(B)
        else:
            brp = bci = bv = None
        po = None if pivot_order is None else np.ascontiguousarray(pivot_order, dtype=np.int32)
        check(lib().hsg_analyze(self._h, n, _ptr(arp), _ptr(aci), _ptr(av), _ptr(brp), _ptr(bci), _ptr(bv),
                                float(alpha), float(beta), _ptr(po)))
        self.n = n

    def estimate(self) -> dict:
        e = _Estimate()
        check(lib().hsg_estimate(self._h, ctypes.byref(e)))
        return {f: getattr(e, f) for f, _ in _Estimate._fields_}

    def factorize(self, alpha, beta) -> bool:
        c = _Inertia()
        check(lib().hsg_factorize(self._h, float(alpha), float(beta), ctypes.byref(c)))
        return bool(c.valid)

    def count(self, alpha, beta, null_pivot_detection=True) -> Inertia:
        c = _Inertia()
        check(lib().hsg_count(self._h, float(alpha), float(beta), int(null_pivot_detection), ctypes.byref(c)))
        return _inertia(c)

    def inertia(self) -> Inertia:
        c = _Inertia()
        check(lib().hsg_inertia(self._h, ctypes.byref(c)))
        return _inertia(c)

    def solve(self, b):
        """Returns K^{-1} b (b: (n,) or (n, p) host array)."""
        x = np.array(b, dtype=np.float64, order="F", copy=True)
        two_d = x.ndim == 2
        if not two_d:
            x = x.reshape(-1, 1, order="F")
        check(lib().hsg_solve(self._h, _ptr(x), x.shape[1], x.shape[0], 0))
        return x if two_d else x[:, 0]

    def solve_device(self, ptr: int, nrhs: int, ld: int):
        """In-place solve of a device buffer (e.g. a torch.cuda tensor's data_ptr())."""
        check(lib().hsg_solve(self._h, ctypes.c_void_p(ptr), nrhs, ld, 1))

    def solve_static(self, ptr: int, nrhs: int, ld: int):
        """In-place solve of a device buffer that allocates no device memory (hsg_solve_static):
        for callers that cannot call cudaMalloc; see include/hsg.h for the size limit."""
        check(lib().hsg_solve_static(self._h, ctypes.c_void_p(ptr), nrhs, ld))

    def release_factors(self) -> bool:
        r = ctypes.c_int32()
        check(lib().hsg_release(self._h, ctypes.byref(r)))
        return bool(r.value)

    def set_null_pivot_detection(self, on: bool):
        check(lib().hsg_set_null_pivot_detection(self._h, int(on)))

    def pivot_order(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.int32)
        check(lib().hsg_pivot_order(self._h, _ptr(out)))
        return out

    def order(self) -> int:
        return int(lib().hsg_order(self._h))


def csr_inspect(m):
    """hsg_csr_inspect on a real CSR matrix (host threads; the interpreter lock is released meanwhile):
    (sorted without duplicates, explicit zero stored, structurally symmetric, entries above / below
    the diagonal, ||M - M^T||_F / ||M||_F, (M + M^T) / 2 on M's pattern or None when M is symmetric)."""
    n = m.shape[0]
    rp = np.ascontiguousarray(m.indptr, dtype=np.int64)
    ci = np.ascontiguousarray(m.indices, dtype=np.int32)
    v = np.ascontiguousarray(m.data, dtype=np.float64)
    flags = np.zeros(3, dtype=np.int32)
    counts = np.zeros(2, dtype=np.int64)
    defect = ctypes.c_double()
    check(lib().hsg_csr_inspect(n, _ptr(rp), _ptr(ci), _ptr(v), _ptr(flags), _ptr(counts), ctypes.byref(defect),
                                None))
    sym = None
    if flags[0] and flags[2] and defect.value > 0:  # a second pass forms (M + M^T) / 2
        sym = np.empty(v.size)
        check(lib().hsg_csr_inspect(n, _ptr(rp), _ptr(ci), _ptr(v), _ptr(flags), _ptr(counts),
                                    ctypes.byref(defect), _ptr(sym)))
    return bool(flags[0]), bool(flags[1]), bool(flags[2]), int(counts[0]), int(counts[1]), defect.value, sym


def compute_ordering(A, seed: int = 2026) -> np.ndarray:
    """hs::compute_ordering: 1-based pivot position of every variable (nested dissection)."""
    rp, ci, _ = upper_csr(A)
    out = np.zeros(A.shape[0], dtype=np.int32)
    check(lib().hsg_compute_ordering(A.shape[0], _ptr(rp), _ptr(ci), seed, _ptr(out)))
    return out


def symbolic_stats(A, pivot_order=None, amalgamate=True) -> dict:
    rp, ci, _ = upper_csr(A)
    e = _Estimate()
    po = None if pivot_order is None else np.ascontiguousarray(pivot_order, dtype=np.int32)
    check(lib().hsg_symbolic_stats(A.shape[0], _ptr(rp), _ptr(ci), _ptr(po), int(amalgamate), ctypes.byref(e)))
    return {f: getattr(e, f) for f, _ in _Estimate._fields_}


class DeviceCsr:
    """A full (both triangles) CSR matrix copied to the current CUDA device for hsg_spmm /
    hsg_shifted_residual; the device arrays are torch tensors (allocation only)."""

    def __init__(self, m, device: str = "cuda:0"):
        import scipy.sparse as sp
        import torch

        m = sp.csr_matrix(m, dtype=np.float64)
        m.sum_duplicates()
        m.sort_indices()
        self.n = m.shape[0]
        self.rp = torch.from_numpy(np.ascontiguousarray(m.indptr, dtype=np.int64)).to(device)
        self.ci = torch.from_numpy(np.ascontiguousarray(m.indices, dtype=np.int32)).to(device)
        self.v = torch.from_numpy(np.ascontiguousarray(m.data, dtype=np.float64)).to(device)

    def ptrs(self):
        return ctypes.c_void_p(self.rp.data_ptr()), ctypes.c_void_p(self.ci.data_ptr()), ctypes.c_void_p(self.v.data_ptr())


def spmm_device(a: DeviceCsr, x, y, alpha: float = 1.0, beta: float = 0.0) -> None:
    """y = alpha A x + beta y with x, y column-major device tensors (torch, shape (p, ld))."""
    p, ldx = x.shape
    check(lib().hsg_spmm(a.n, *a.ptrs(), ctypes.c_void_p(x.data_ptr()), ldx, ctypes.c_void_p(y.data_ptr()), y.shape[1],
                         p, float(alpha), float(beta)))


def shifted_residual_device(a: DeviceCsr, b, sigma: float, x, y, r, omega=None) -> None:
    """r = B x - (A y - sigma B y) and omega (per column) on device tensors of shape (p, ld);
    b None: B = I."""
    p = x.shape[0]
    bp = b.ptrs() if b is not None else (None, None, None)
    check(lib().hsg_shifted_residual(a.n, *a.ptrs(), *bp, float(sigma), ctypes.c_void_p(x.data_ptr()), x.shape[1],
                                     ctypes.c_void_p(y.data_ptr()), y.shape[1],
                                     None if r is None else ctypes.c_void_p(r.data_ptr()),
                                     a.n if r is None else r.shape[1], p,
                                     None if omega is None else ctypes.c_void_p(omega.data_ptr())))


def clear_analysis_cache() -> None:
    """Empties the process-wide analysis cache (the next solve on any pattern analyses afresh)."""
    check(lib().hsg_clear_analysis_cache())


def kernel_launches() -> int:
    """Kernel launches this library has issued in the process so far."""
    return int(lib().hsg_kernel_launches())


def fp64_peak_tflops(device: int = 0) -> float:
    """Measured FP64 FMA throughput (TFLOP/s) of the device."""
    v = ctypes.c_double()
    check(lib().hsg_fp64_peak_probe(device, ctypes.byref(v)))
    return float(v.value)
