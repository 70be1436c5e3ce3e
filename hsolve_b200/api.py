"""hsolve.solve(...) on the B200 path (hsolve python/hsolve/__init__.py:347-419): same signature,
argument handling, configuration merging and error classes; the work runs in the native library
through the C ABI of include/hsg_solve.h (hsg_eigsolve)."""
from __future__ import annotations

import ctypes
import json
import numbers
import operator
import os
import warnings
from dataclasses import dataclass
from typing import Any

import numpy as np

from . import _native
from .errors import HsolveIOError, HsolveWarning, InvalidInputError, NotHermitianError, UnsupportedError


class _SolveConfig(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int32), ("sigma", ctypes.c_double), ("k", ctypes.c_int64),
                ("lower", ctypes.c_double), ("upper", ctypes.c_double), ("problem", ctypes.c_int32),
                ("tol", ctypes.c_double), ("inner_tol_factor", ctypes.c_double), ("ncv", ctypes.c_int64),
                ("block_size", ctypes.c_int32), ("slice_size", ctypes.c_int64), ("max_restarts", ctypes.c_int32),
                ("seed", ctypes.c_uint64), ("certificate", ctypes.c_int32), ("max_shift_retries", ctypes.c_int32),
                ("factor_precision", ctypes.c_int32), ("device", ctypes.c_int32), ("verbose", ctypes.c_int32),
                ("batch_shifts", ctypes.c_int32), ("complex_tol", ctypes.c_double),
                ("zero_filter_tol", ctypes.c_double)]


_P = ctypes.c_void_p
_SOLVE_SIGS = {
    "hsg_default_solve_config": (None, [_P]),
    "hsg_eigsolve": (ctypes.c_int, [ctypes.c_int64, _P, _P, _P, _P, _P, _P, _P, _P]),
    "hsg_solution_sizes": (ctypes.c_int, [_P, _P, _P]),
    "hsg_solution_copy": (ctypes.c_int, [_P, _P, _P]),
    "hsg_solution_complex_count": (ctypes.c_int, [_P, _P]),
    "hsg_solution_complex_copy": (ctypes.c_int, [_P, _P, _P]),
    "hsg_solution_report": (ctypes.c_char_p, [_P]),
    "hsg_solution_free": (None, [_P]),
    "hsg_session_create": (ctypes.c_int, [ctypes.c_int64, _P, _P, _P, _P, _P, _P, ctypes.c_int32, ctypes.c_uint64, _P]),
    "hsg_session_solve": (ctypes.c_int, [_P, _P, _P]),
    "hsg_session_free": (None, [_P]),
    "hsg_session_estimate": (ctypes.c_int, [_P, _P]),
    "hsg_default_exclusion_options": (None, [_P]),
    "hsg_session_exclusion_check": (ctypes.c_int, [_P, _P, ctypes.c_int64, ctypes.c_int64, _P, _P]),
    "hsg_exclusion_failure_bound": (ctypes.c_double, [ctypes.c_double, ctypes.c_int64, ctypes.c_int64,
                                                      ctypes.c_int64, ctypes.c_double, ctypes.c_int32]),
    "hsg_exclusion_block_steps": (ctypes.c_int64, [ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                                                   ctypes.c_int64, ctypes.c_double, ctypes.c_int32]),
}
_native.SIGNATURES.update(_SOLVE_SIGS)


class _ExclusionOptions(ctypes.Structure):
    """hsg_exclusion_options_t (include/hsg_solve.h)."""
    _fields_ = [("sigma", ctypes.c_double), ("radius", ctypes.c_double), ("pass_radius", ctypes.c_double),
                ("delta", ctypes.c_double), ("block_size", ctypes.c_int32), ("max_block_steps", ctypes.c_int32),
                ("max_krylov_vectors", ctypes.c_int32), ("pad", ctypes.c_int32), ("seed", ctypes.c_uint64),
                ("kappa", ctypes.c_double), ("rounding_margin", ctypes.c_double)]


class _ExclusionResult(ctypes.Structure):
    """hsg_exclusion_result_t (include/hsg_solve.h)."""
    _fields_ = [("status", ctypes.c_int32), ("exact", ctypes.c_int32), ("over_budget", ctypes.c_int32),
                ("rigorous", ctypes.c_int32), ("sigma", ctypes.c_double), ("claim_threshold", ctypes.c_double),
                ("pass_threshold", ctypes.c_double), ("coupling", ctypes.c_double), ("epsilon", ctypes.c_double),
                ("kappa", ctypes.c_double), ("deflated", ctypes.c_int64), ("dimension", ctypes.c_int64),
                ("found_inside", ctypes.c_int64), ("certified_inside", ctypes.c_int64),
                ("block_size", ctypes.c_int64), ("block_steps_planned", ctypes.c_int64),
                ("block_steps", ctypes.c_int64), ("krylov_vectors_planned", ctypes.c_int64),
                ("max_ritz", ctypes.c_double), ("failure_probability", ctypes.c_double),
                ("new_count", ctypes.c_int64), ("new_inside", ctypes.c_int64), ("op_applications", ctypes.c_int64),
                ("setup_s", ctypes.c_double), ("krylov_s", ctypes.c_double)]


_EXCLUSION_STATUS = {0: "passed", 1: "detected", 2: "inconclusive"}

_MODES = ("nearest", "interval", "smallest", "largest")
_STORAGES = ("auto", "full", "upper", "lower")
_PROBLEMS = ("auto", "standard", "generalized_definite", "generalized_indefinite")
_PRECISIONS = ("double", "single", "auto")
_CERTS = ("exact", "randomized", "auto", "off")
# SolverConfig keys (include/hsolve/solver.hpp:71-235): all are accepted; the ones this path does not
# act on are validated for type only and reported as ignored.
_KNOWN_KEYS = {"target", "problem", "method", "tol", "hermitian_tol", "inner_tol_factor", "ncv", "block_size",
               "slice_size", "max_restarts", "seed", "threads", "memory_budget_gb", "factor_precision", "ordering",
               "deterministic", "blr", "out_of_core", "inertia_check", "inertia_counter", "certificate",
               "certificate_delta", "certificate_fault_drop", "inexact_fault_reject", "certificate_fault_count",
               "structure_candidates", "subspace_bound", "secure", "zero_filter_tol", "complex_tol",
               "max_shift_retries", "device", "batch_shifts"}


@dataclass(repr=False, eq=False)
class SolveResult:
    """Result of solve(): same fields as hsolve.SolveResult (python/hsolve/__init__.py:141-170)."""

    eigenvalues: np.ndarray
    eigenvectors: np.ndarray
    complex_eigenvalues: np.ndarray
    complex_eigenvectors: np.ndarray
    report: dict
    config: dict

    @property
    def success(self) -> bool:
        return bool(self.report.get("success", False))

    def __repr__(self) -> str:
        return (f"SolveResult(n={self.eigenvectors.shape[0]}, eigenvalues={self.eigenvalues.size}, "
                f"complex_eigenvalues={self.complex_eigenvalues.size}, problem={self.report.get('problem')!r}, "
                f"success={self.success})")


class _Default:
    __slots__ = ("value",)

    def __init__(self, value):
        self.value = value

    def __repr__(self):
        return repr(self.value)


def _real(x: Any, name: str) -> float:
    if isinstance(x, np.ndarray) and x.ndim == 0 and x.dtype.kind in "iuf":
        return float(x)
    if isinstance(x, (bool, np.bool_)) or not isinstance(x, numbers.Real):
        raise TypeError(f"{name} must be a real number, got {type(x).__name__}")
    return float(x)


def _integer(x: Any, name: str) -> int:
    if isinstance(x, (bool, np.bool_)):
        raise TypeError(f"{name} must be an integer, got bool")
    try:
        return operator.index(x)
    except TypeError as e:
        raise TypeError(f"{name} must be an integer, got {type(x).__name__}") from e


def _read_config(config) -> dict:
    if config is None:
        return {}
    if isinstance(config, dict):
        return json.loads(json.dumps(config, default=lambda o: o.item() if isinstance(o, np.generic) else str(o)))
    if isinstance(config, (str, bytes, os.PathLike)):
        path = os.fsdecode(config)
        try:
            with open(path, encoding="utf-8") as f:
                text = f.read()
        except OSError as e:
            raise HsolveIOError(f"cannot read config file {path}: {e}") from e
        try:
            doc = json.loads(text)
        except json.JSONDecodeError as e:
            raise InvalidInputError(f"config file {path}: invalid JSON: {e}") from None
        if not isinstance(doc, dict):
            raise InvalidInputError(f"config file {path}: top level must be a JSON object")
        return doc
    raise TypeError(f"config must be a dict, a path to config.json or None, got {type(config).__name__}")


def merge_config(config, sigma, k, mode, lower, upper, tol, threads) -> dict:
    """Keyword arguments override the config document (python/hsolve/__init__.py:231-275)."""
    cfg = _read_config(config)
    unknown = set(cfg) - _KNOWN_KEYS
    if unknown:
        raise InvalidInputError(f"config: unknown key(s) {sorted(unknown)}")
    target = cfg.get("target", {})
    if not isinstance(target, dict):
        raise InvalidInputError("config: 'target' must be an object")
    target = dict(target)
    explicit_mode = not isinstance(mode, _Default)
    interval_bounds = lower is not None or upper is not None
    if explicit_mode:
        if not isinstance(mode, str):
            raise TypeError(f"mode must be a string, got {type(mode).__name__}")
        if mode not in _MODES:
            raise InvalidInputError(f"mode = {mode!r} is not one of {_MODES}")
        target["mode"] = mode
    elif interval_bounds:
        if sigma is not None:
            raise InvalidInputError("give sigma (nearest) or lower/upper (interval), not both, or pass mode=")
        target["mode"] = "interval"
    elif sigma is not None:
        target["mode"] = "nearest"
    if sigma is not None:
        target["sigma"] = _real(sigma, "sigma")
    if lower is not None:
        target["lower"] = _real(lower, "lower")
    if upper is not None:
        target["upper"] = _real(upper, "upper")
    if not isinstance(k, _Default):
        target["k"] = _integer(k, "k")
    cfg["target"] = target
    if not isinstance(tol, _Default):
        cfg["tol"] = _real(tol, "tol")
    if not isinstance(threads, _Default):
        cfg["threads"] = _integer(threads, "threads")
    try:  # the config is a JSON document: no inf / nan anywhere in it
        json.dumps(cfg, allow_nan=False)
    except ValueError as e:
        raise InvalidInputError(f"config: {e} (JSON has no inf/nan)") from None
    return cfg


def _struct_from(cfg: dict, verbose: int) -> _SolveConfig:
    c = _SolveConfig()
    _native.lib().hsg_default_solve_config(ctypes.byref(c))
    t = cfg.get("target", {})
    mode = t.get("mode", "nearest")
    if mode not in _MODES:
        raise InvalidInputError(f"target.mode = {mode!r} is not one of {_MODES}")
    c.mode = _MODES.index(mode)
    c.sigma = float(t.get("sigma", 0.0))
    c.k = int(t.get("k", 6))
    c.lower = float(t.get("lower", 0.0))
    c.upper = float(t.get("upper", 0.0))
    prob = cfg.get("problem", "auto")
    if prob not in _PROBLEMS:
        raise InvalidInputError(f"problem = {prob!r} is not one of {_PROBLEMS}")
    c.problem = _PROBLEMS.index(prob)
    c.tol = float(cfg.get("tol", 1e-10))
    c.inner_tol_factor = float(cfg.get("inner_tol_factor", 0.1))
    c.ncv = int(cfg.get("ncv", 0))
    c.block_size = int(cfg.get("block_size", 0))
    c.slice_size = int(cfg.get("slice_size", 0))
    c.max_restarts = int(cfg.get("max_restarts", 1000))
    c.seed = int(cfg.get("seed", 2026))
    cert = cfg.get("certificate", "exact")
    if cert not in _CERTS:
        raise InvalidInputError(f"certificate = {cert!r} is not one of {_CERTS}")
    c.certificate = 3 if cert == "off" or cfg.get("inertia_check", "auto") == "off" else 0
    c.max_shift_retries = int(cfg.get("max_shift_retries", 5))
    prec = cfg.get("factor_precision", "double")
    if prec not in _PRECISIONS:
        raise InvalidInputError(f"factor_precision = {prec!r} is not one of {_PRECISIONS}")
    c.factor_precision = 1 if prec == "single" else 0
    c.device = int(cfg.get("device", 0))
    c.verbose = int(verbose)
    c.batch_shifts = 1 if bool(cfg.get("batch_shifts", True)) else 0
    c.complex_tol = float(cfg.get("complex_tol", 1e-8))
    c.zero_filter_tol = float(cfg.get("zero_filter_tol", -1.0))
    if not (0.0 < c.tol < 1.0):
        raise InvalidInputError("tol must be in (0, 1)")
    return c


def _is_csr(m) -> bool:
    import scipy.sparse as sp

    return sp.issparse(m) and m.format == "csr"


def _as_csr(m, name, storage):
    import scipy.sparse as sp

    if isinstance(m, (str, bytes, os.PathLike)):
        path = os.fsdecode(m)
        if path.endswith(".npz"):
            m = sp.load_npz(path)
        elif path.endswith(".npy"):
            m = np.load(path)
        elif path.endswith(".mtx"):
            import scipy.io

            m = scipy.io.mmread(path)
        else:
            raise HsolveIOError(f"{name}: unsupported file type {path}")
    if hasattr(m, "matvec") and not isinstance(m, np.ndarray) and not sp.issparse(m):
        raise TypeError(f"{name}: hsolve factorizes the matrix and needs its entries, not a LinearOperator")
    if not sp.issparse(m):
        arr = np.asarray(m)
        if arr.dtype == object or arr.ndim != 2:
            raise InvalidInputError(f"{name}: expected a 2-D numeric matrix")
        m = sp.csr_matrix(arr)
    m = sp.csr_matrix(m)
    if m.shape[0] != m.shape[1]:
        raise InvalidInputError(f"{name}: matrix must be square, got {m.shape}")
    if np.iscomplexobj(m.data):
        m = sp.csr_matrix(m, dtype=np.complex128)
        if not np.any(m.data.imag != 0):
            m = sp.csr_matrix(m.real)  # solved as real; the eigenvectors still come back complex
    else:
        m = sp.csr_matrix(m, dtype=np.float64)
    # the caller's matrix is never modified: copy before any in-place clean-up
    copied = False
    if not m.has_canonical_format:
        m = m.copy()
        copied = True
        m.sum_duplicates()
    if m.nnz and not np.all(m.data):
        if not copied:
            m = m.copy()
        m.eliminate_zeros()
    if storage == "upper":
        m = sp.triu(m) + sp.triu(m, 1).conj().T
    elif storage == "lower":
        m = sp.tril(m) + sp.tril(m, -1).conj().T
    elif storage == "auto":
        # entries strictly above / below the diagonal, counted on the CSR arrays
        rows = np.repeat(np.arange(m.shape[0], dtype=m.indices.dtype), np.diff(m.indptr))
        up = int(np.count_nonzero(m.indices > rows))
        lo = int(np.count_nonzero(m.indices < rows))
        if (up == 0) != (lo == 0):
            m = sp.triu(m) + sp.triu(m, 1).conj().T if lo == 0 else sp.tril(m) + sp.tril(m, -1).conj().T
    m = sp.csr_matrix(m)
    if not m.has_canonical_format:
        m.sum_duplicates()
    m.sort_indices()
    return m


def _complex_dtype(m) -> bool:
    """True when the input's value type is complex (the eigenvectors are then returned complex)."""
    import scipy.sparse as sp

    if isinstance(m, (str, bytes, os.PathLike)):
        path = os.fsdecode(m)
        try:
            if path.endswith(".npz"):
                return np.iscomplexobj(sp.load_npz(path).data)
            if path.endswith(".npy"):
                return np.iscomplexobj(np.load(path, mmap_mode="r"))
            if path.endswith(".mtx"):
                import scipy.io

                return scipy.io.mminfo(path)[4] == "complex"
        except Exception:
            return False
        return False
    if sp.issparse(m):
        return np.iscomplexobj(m.data)
    return np.iscomplexobj(np.asarray(m))


def _prepare(m, name, storage, tol):
    """The input as a canonical CSR matrix holding both triangles, symmetrized, with its Hermitian
    defect: _as_csr + _hermitian_check. A real CSR matrix that is already canonical (sorted, no
    duplicates, no stored zeros), holds both triangles and is structurally symmetric is checked by
    the native hsg_csr_inspect on host threads, outside the interpreter lock; every other input takes
    the general path."""
    import scipy.sparse as sp

    if (storage == "auto" and sp.issparse(m) and m.format == "csr" and m.dtype == np.float64 and m.ndim == 2
            and m.shape[0] == m.shape[1] and m.nnz > 0 and m.indices.dtype in (np.int32, np.int64)
            and m.shape[0] < 2**31):
        canonical, zero, symmetric, up, lo, defect, sym = _native.csr_inspect(m)
        if canonical and not zero and symmetric and (up == 0) == (lo == 0):
            if defect > tol:
                raise NotHermitianError(f"{name}: ||M - M^H||_F / ||M||_F = {defect:.3e} > hermitian_tol = {tol:g}")
            if defect > 0:
                m = sp.csr_matrix((sym, m.indices.copy(), m.indptr.copy()), shape=m.shape)
            return m, defect
    return _hermitian_check(_as_csr(m, name, storage), name, tol)


def _hermitian_check(m, name, tol):
    """||M - M^H||_F / ||M||_F of a canonical CSR matrix (sorted, no duplicates); raises
    NotHermitianError above tol, else returns (M + M^H) / 2 (M itself when the defect is 0) and the
    defect. With a structurally symmetric pattern M^H has M's index arrays, and the defect is an
    entrywise difference of the two value arrays."""
    import scipy.sparse as sp

    t = m.T.tocsr()
    t.sort_indices()
    same = np.array_equal(t.indptr, m.indptr) and np.array_equal(t.indices, m.indices)
    if same:
        th = t.data.conj() if np.iscomplexobj(t.data) else t.data
        dd = m.data - th
    else:
        dd = (m - m.conj().T).data
    nrm = float(np.sqrt(np.vdot(m.data, m.data).real))
    defect = float(np.sqrt(np.vdot(dd, dd).real)) / nrm if nrm > 0 else 0.0
    if defect > tol:
        raise NotHermitianError(f"{name}: ||M - M^H||_F / ||M||_F = {defect:.3e} > hermitian_tol = {tol:g}")
    if defect > 0:
        if same:
            m = sp.csr_matrix(((m.data + th) * 0.5, m.indices.copy(), m.indptr.copy()), shape=m.shape)
        else:
            m = ((m + m.conj().T) * 0.5).tocsr()
            m.sort_indices()
    return m, defect


def _embed(m):
    """Real symmetric 2n x 2n embedding [[Re M, -Im M], [Im M, Re M]] of a Hermitian matrix M (the
    reference's complex path, src/factor/mumps_input.cpp:44-150): every eigenvalue of the pencil
    appears twice and every inertia count doubles."""
    import scipy.sparse as sp

    x = sp.csr_matrix(m.real)
    y = sp.csr_matrix(m.imag) if np.iscomplexobj(m.data) else sp.csr_matrix(m.shape)
    e = sp.bmat([[x, -y], [y, x]], format="csr")
    e.eliminate_zeros()
    e.sort_indices()
    return e


def _unembed(w, v, report, a, b, tol, mode, sigma, k):
    """Complex eigenpairs of the Hermitian pencil (a, b) from the solution (w, v) of its embedding:
    each cluster of equal embedded eigenvalues (2m of them) spans an m-dimensional complex
    eigenspace, recovered B-orthonormal from the vectors u + i v of the embedded pairs [u; v] and
    a Rayleigh-Ritz step within the cluster. Counts of the certificate are halved; an odd count
    means the embedding's inertia split was not even and the certificate fails."""
    n = a.shape[0]
    scale = float(report.get("scale", 0.0)) or 1.0
    order = np.argsort(w, kind="stable")
    ws, vs = w[order], v[:, order]
    clusters, i = [], 0
    while i < ws.size:
        j = i + 1
        while j < ws.size and abs(ws[j] - ws[j - 1]) <= 1e-8 * (abs(ws[j]) + scale):
            j += 1
        clusters.append((i, j))
        i = j
    lam, vecs, odd = [], [], False
    bmul = (lambda z: b @ z) if b is not None else (lambda z: z)
    for i, j in clusters:
        z = vs[:n, i:j] + 1j * vs[n:, i:j]
        s = j - i
        m = s // 2
        odd = odd or s % 2 == 1
        if m == 0:
            continue
        g = z.conj().T @ bmul(z)
        g = 0.5 * (g + g.conj().T)
        gv, gq = np.linalg.eigh(g)
        gv, gq = gv[-m:], gq[:, -m:]
        x = z @ (gq / np.sqrt(np.maximum(gv, np.finfo(float).tiny)))
        h = x.conj().T @ (a @ x)
        hv, hq = np.linalg.eigh(0.5 * (h + h.conj().T))
        lam.extend(hv.tolist())
        vecs.append(x @ hq)
    lam = np.asarray(lam, dtype=np.float64)
    x = np.hstack(vecs) if vecs else np.zeros((n, 0), dtype=np.complex128)
    if mode == "nearest":
        o = np.argsort(np.abs(lam - sigma), kind="stable")[:k]
    elif mode == "smallest":
        o = np.argsort(lam, kind="stable")[:k]
    elif mode == "largest":
        o = np.argsort(-lam, kind="stable")[:k]
    else:
        o = np.argsort(lam, kind="stable")
    lam, x = lam[o], np.asfortranarray(x[:, o])
    na, nb = float(report.get("norm2_a", 0.0)), float(report.get("norm2_b", 1.0)) or 1.0
    pairs = []
    for q in range(lam.size):
        r = a @ x[:, q] - lam[q] * bmul(x[:, q])
        rn, xn = float(np.linalg.norm(r)), float(np.linalg.norm(x[:, q]))
        eta = rn / ((na + abs(lam[q]) * nb) * xn) if xn > 0 else np.inf
        pairs.append({"lambda_re": float(lam[q]), "lambda_im": 0.0, "abs_residual": rn,
                      "rel_residual": rn / (abs(lam[q]) * xn) if lam[q] != 0 and xn > 0 else rn,
                      "backward_error": eta, "accepted": bool(eta <= tol)})
    rep = dict(report)
    rep["n"] = n
    rep["complex_scalars"] = True
    rep["embedding"] = {"order": 2 * n, "embedded_eigenvalues": int(w.size), "odd_cluster": bool(odd)}
    rep["pairs"] = pairs
    cert = dict(rep.get("certificate", {}))
    passed = bool(cert.get("passed", True)) and not odd
    for key in ("count_inertia", "count_found"):
        if key in cert and cert[key] is not None and cert[key] >= 0:
            passed = passed and cert[key] % 2 == 0
            cert[key] = cert[key] // 2
    if cert:
        cert["passed"] = passed
        rep["certificate"] = cert
    if "slices" in rep:
        sl = []
        for r0 in rep["slices"]:
            r1 = dict(r0)
            for key in ("count", "count_found", "count_inertia"):
                if isinstance(r1.get(key), int):
                    r1[key] //= 2
            sl.append(r1)
        rep["slices"] = sl
    ok = all(p["accepted"] for p in pairs) and (not cert or cert["passed"])
    if mode == "interval" and cert.get("count_inertia") is not None:
        ok = ok and lam.size == cert["count_inertia"]
    if mode in ("nearest", "smallest", "largest"):
        ok = ok and lam.size == k
    rep["success"] = bool(ok)
    return lam, x, rep


def solve(A, B=None, *, sigma=None, k=_Default(6), mode=_Default("nearest"), lower=None, upper=None,
          tol=_Default(1e-10), config=None, threads=_Default(0), verbose: int = 0, storage: str = "auto"):
    """Solve A x = lambda B x (B=None: A x = lambda x) for Hermitian A, B with B positive definite,
    on the GPU: the nearest-k target around sigma or all eigenvalues in [lower, upper], each with the
    exact Sylvester-inertia completeness certificate (hsolve.solve's contract). Real symmetric input
    is factorized directly; complex Hermitian input goes through the real 2n embedding
    [[Re, -Im], [Im, Re]] (as the reference does) and comes back as complex eigenvectors."""
    if storage not in _STORAGES:
        raise InvalidInputError(f"storage = {storage!r} is not one of {_STORAGES}")
    cfg = merge_config(config, sigma, k, mode, lower, upper, tol, threads)
    verbose = _integer(verbose, "verbose")
    cdtype = _complex_dtype(A) or (B is not None and _complex_dtype(B))
    htol = float(cfg.get("hermitian_tol", 1e-10))
    a, da = _prepare(A, "A", storage, htol)
    b = None
    db = 0.0
    if B is not None:
        b = _as_csr(B, "B", storage) if not _is_csr(B) else B
        if b.shape != a.shape:
            raise InvalidInputError(f"A is {a.shape} but B is {b.shape}")
        b, db = _prepare(b, "B", storage, htol)
    if np.iscomplexobj(a.data) or (b is not None and np.iscomplexobj(b.data)):
        ae, be = _embed(a), (_embed(b) if b is not None else None)
        w, v, report, _ = _eigsolve(ae, be, _struct_from(_embedded_config(cfg), verbose))
        return _complex_result(w, v, report, a, b, cfg, da, db)
    w, v, report, cplx = _eigsolve(a, b, _struct_from(cfg, verbose))
    return _finish(w, v, report, cfg, da, db, cdtype, cplx)


def _embedded_config(cfg: dict) -> dict:
    """The config of the embedded (2n real) problem: twice the requested number of pairs."""
    ce = json.loads(json.dumps(cfg))
    t = ce.setdefault("target", {})
    if t.get("mode", "nearest") in ("nearest", "smallest", "largest"):
        t["k"] = 2 * int(t.get("k", 6))
    return ce


def _complex_result(w, v, report, a, b, cfg, da, db) -> SolveResult:
    t = cfg.get("target", {})
    mode = t.get("mode", "nearest")
    lam, x, rep = _unembed(w, v, report, a, b, float(cfg.get("tol", 1e-10)), mode, float(t.get("sigma", 0.0)),
                           int(t.get("k", 6)))
    rep["hermitian_defect_a"] = da
    rep["hermitian_defect_b"] = db
    result = SolveResult(lam, x, np.zeros(0, dtype=np.complex128), np.zeros((a.shape[0], 0), dtype=np.complex128),
                         rep, cfg)
    if not result.success:
        warnings.warn("hsolve: the solve finished without meeting the tolerance (see result.report['pairs'] "
                      "and result.report['warnings'])", HsolveWarning, stacklevel=3)
    return result


def _eigsolve(a, b, c):
    """hsg_eigsolve on real symmetric CSR matrices: (eigenvalues, eigenvectors, report)."""
    n = a.shape[0]
    arp = np.ascontiguousarray(a.indptr, dtype=np.int64)
    aci = np.ascontiguousarray(a.indices, dtype=np.int32)
    av = np.ascontiguousarray(a.data, dtype=np.float64)
    if b is not None:
        brp = np.ascontiguousarray(b.indptr, dtype=np.int64)
        bci = np.ascontiguousarray(b.indices, dtype=np.int32)
        bv = np.ascontiguousarray(b.data, dtype=np.float64)
    else:
        brp = bci = bv = None
    lib = _native.lib()
    h = ctypes.c_void_p()
    p = _native._ptr
    _native.check(lib.hsg_eigsolve(n, p(arp), p(aci), p(av), p(brp), p(bci), p(bv), ctypes.byref(c), ctypes.byref(h)))
    return _fetch(h)


def _fetch(h):
    """(eigenvalues, eigenvectors, report, (complex eigenvalues, complex eigenvectors)) of a native
    solution handle, which is freed."""
    lib = _native.lib()
    p = _native._ptr
    try:
        nn, m, mc = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _native.check(lib.hsg_solution_sizes(h, ctypes.byref(nn), ctypes.byref(m)))
        w = np.zeros(m.value)
        v = np.zeros((nn.value, m.value), order="F")
        _native.check(lib.hsg_solution_copy(h, p(w), p(v)))
        _native.check(lib.hsg_solution_complex_count(h, ctypes.byref(mc)))
        cw = np.zeros(mc.value, dtype=np.complex128)
        cv = np.zeros((nn.value, mc.value), dtype=np.complex128, order="F")
        if mc.value:
            _native.check(lib.hsg_solution_complex_copy(h, p(cw), p(cv)))
        report = json.loads(lib.hsg_solution_report(h).decode())
    finally:
        lib.hsg_solution_free(h)
    return w, v, report, (cw, cv)


def _finish(w, v, report, cfg, da, db, complex_vectors=False, cplx=None) -> SolveResult:
    n = v.shape[0]
    report["hermitian_defect_a"] = da
    report["hermitian_defect_b"] = db
    if complex_vectors:
        v = np.asfortranarray(v.astype(np.complex128))
    cw, cv = cplx if cplx is not None else (np.zeros(0, dtype=np.complex128), np.zeros((n, 0), dtype=np.complex128))
    result = SolveResult(w, v, cw, cv, report, cfg)
    if not result.success:
        warnings.warn("hsolve: the solve finished without meeting the tolerance (see result.report['pairs'] "
                      "and result.report['warnings'])", HsolveWarning, stacklevel=3)
    return result


class Session:
    """A pencil (A, B) resident on the GPU with its nested-dissection analysis and norm bounds done
    once; solve(...) takes solve()'s target arguments and reuses them for every target and shift
    (the serving path's symbolic reuse)."""

    def __init__(self, A, B=None, *, device: int = 0, seed: int = 2026, storage: str = "auto",
                 hermitian_tol: float = 1e-10):
        self._cdtype = _complex_dtype(A) or (B is not None and _complex_dtype(B))
        a, self._da = _prepare(A, "A", storage, hermitian_tol)
        self._db = 0.0
        b = None
        if B is not None:
            b = _as_csr(B, "B", storage) if not _is_csr(B) else B
            if b.shape != a.shape:
                raise InvalidInputError(f"A is {a.shape} but B is {b.shape}")
            b, self._db = _prepare(b, "B", storage, hermitian_tol)
        self._complex = None
        if np.iscomplexobj(a.data) or (b is not None and np.iscomplexobj(b.data)):
            self._complex = (a, b)  # kept for the eigenvectors; the session holds the embedding
            a, b = _embed(a), (_embed(b) if b is not None else None)
        self.n = a.shape[0]
        self.device = device
        keep = [np.ascontiguousarray(a.indptr, dtype=np.int64), np.ascontiguousarray(a.indices, dtype=np.int32),
                np.ascontiguousarray(a.data, dtype=np.float64)]
        if b is not None:
            keep += [np.ascontiguousarray(b.indptr, dtype=np.int64), np.ascontiguousarray(b.indices, dtype=np.int32),
                     np.ascontiguousarray(b.data, dtype=np.float64)]
        else:
            keep += [None, None, None]
        p = _native._ptr
        h = ctypes.c_void_p()
        _native.check(_native.lib().hsg_session_create(self.n, *[p(x) for x in keep], int(device), int(seed),
                                                       ctypes.byref(h)))
        self._h = h

    def solve(self, *, sigma=None, k=_Default(6), mode=_Default("nearest"), lower=None, upper=None,
              tol=_Default(1e-10), config=None, verbose: int = 0) -> SolveResult:
        cfg = merge_config(config, sigma, k, mode, lower, upper, tol, _Default(0))
        cfg.setdefault("device", self.device)
        c = _struct_from(_embedded_config(cfg) if self._complex else cfg, verbose)
        h = ctypes.c_void_p()
        _native.check(_native.lib().hsg_session_solve(self._h, ctypes.byref(c), ctypes.byref(h)))
        w, v, report, cplx = _fetch(h)
        if self._complex:
            return _complex_result(w, v, report, self._complex[0], self._complex[1], cfg, self._da, self._db)
        return _finish(w, v, report, cfg, self._da, self._db, self._cdtype, cplx)

    def exclusion_check(self, X, *, sigma: float, radius: float, pass_radius: float, delta: float = 1e-12,
                        block_size: int = 4, seed: int = 2026, kappa: float = 1.0, rounding_margin: float = 1e-6,
                        max_block_steps: int = 0, max_krylov_vectors: int = 512) -> dict:
        """Randomized exclusion certificate (hsolve's exclusion_check, include/hsolve/verify.hpp:18-80):
        with X the found eigenvectors (n x m, any basis of their span), does the pencil have more
        eigenvalues than the found ones within `radius` of `sigma`? The session factorizes at sigma, and
        a block Lanczos run on the complement of span X, whose length is fixed beforehand from `delta`,
        decides: status "passed" (no Ritz value with |theta| >= 1 / pass_radius; the statement fails with
        probability <= failure_probability <= delta), "detected" or "inconclusive" (the gap between
        radius and pass_radius is too small for the coupling of X, or the plan exceeds
        max_krylov_vectors). B must be positive definite. For a complex pencil X is complex and the
        check runs on the real 2n embedding (every count doubles)."""
        x = np.asarray(X)
        if x.ndim == 1:
            x = x[:, None]
        if x.ndim != 2:
            raise InvalidInputError(f"X must be an n x m array, got {x.ndim} dimensions")
        if np.iscomplexobj(x) and not self._complex:
            raise InvalidInputError("X is complex but the pencil is real")
        if self._complex:
            xc = x.astype(np.complex128)
            x = np.block([[xc.real, -xc.imag], [xc.imag, xc.real]])
        x = np.asfortranarray(x, dtype=np.float64)
        if x.shape[0] != self.n:
            raise InvalidInputError(f"X has {x.shape[0]} rows, the pencil has {self.n}")
        o = _ExclusionOptions()
        _native.lib().hsg_default_exclusion_options(ctypes.byref(o))
        o.sigma, o.radius, o.pass_radius, o.delta = float(sigma), float(radius), float(pass_radius), float(delta)
        o.block_size, o.seed, o.kappa = int(block_size), int(seed), float(kappa)
        o.rounding_margin, o.max_block_steps, o.max_krylov_vectors = float(rounding_margin), int(max_block_steps), \
            int(max_krylov_vectors)
        r = _ExclusionResult()
        _native.check(_native.lib().hsg_session_exclusion_check(self._h, x.ctypes.data_as(ctypes.c_void_p),
                                                                x.shape[1], x.shape[0], ctypes.byref(o),
                                                                ctypes.byref(r)))
        out = {f: getattr(r, f) for f, _ in _ExclusionResult._fields_}
        out["status"] = _EXCLUSION_STATUS.get(r.status, "inconclusive")
        for key in ("exact", "over_budget", "rigorous"):
            out[key] = bool(out[key])
        return out

    def estimate(self) -> dict:
        """Analysis of the session's pencil (for a complex pencil, of its real 2n embedding): factor
        entries, nnz(L), flops and device memory (MB) of one factorization object."""
        e = _native._Estimate()
        _native.check(_native.lib().hsg_session_estimate(self._h, ctypes.byref(e)))
        return {f: getattr(e, f) for f, _ in _native._Estimate._fields_}

    def close(self):
        if getattr(self, "_h", None):
            _native.lib().hsg_session_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
