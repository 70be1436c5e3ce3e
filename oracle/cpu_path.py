"""ORACLE (test infrastructure and the timed CPU baseline only; never imported by the product path):
a CPU restatement of hsolve's certified shift-invert eigensolve, end to end, on the oracle's
multifrontal LDL^T (oracle/mf_ldlt.c, the restatement of the MUMPS path) - the reference's CPU path
with this project's port standing in for MUMPS, which needs a Fortran compiler that is absent.

It follows the reference's driver at the level of its documented contract, as the GPU driver does:
* interval targets (src/driver/definite.cpp WindowSolver): Sylvester counts nu_-(A - s B) at the
  window ends, with outward endpoint moves on singular shifts (src/driver/steps.cpp:549-571), one
  shift per slice of at most `slice_size` eigenvalues (cut counts split larger windows);
* per slice: block thick-restart Lanczos / Krylov-Schur on OP = (A - sigma B)^{-1} B in the B inner
  product (src/eigen/block_lanczos.cpp:280-322): CGS2 re-orthogonalisation and CholQR2 (block_ortho,
  src/eigen/block_ortho.cpp:165,270), Rayleigh-Ritz on the projected matrix, locking of pairs whose
  coupling is at rounding level (:65), tol_inner = tol * 0.1 (include/hsolve/solver.hpp:78);
* block width p in {1, 2, 4, 8} by the wanted count (solver.hpp:75-108);
* acceptance: eta = ||A x - lambda B x|| / ((||A|| + |lambda| ||B||) ||x||) <= tol with Lanczos
  estimates of the norms (src/driver/projection.cpp:54), certificate: found == counted per slice.

The ordering is the reference's own nested dissection (oracle/_ref, built from the reference's
sources) where that library exists, else this project's (hsolve_b200's host ordering).
"""
from __future__ import annotations

import time

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import ref as refk
from .ldlt import OracleLDLT, threads


def _ordering(pattern):
    """1-based-free pivot order (new -> old) of the pencil pattern."""
    if refk.available():
        perm_in, _ = refk.compute_ordering(pattern)   # PERM_IN: 1-based position of every variable
    else:
        import hsolve_b200 as hs  # noqa: WPS433 - fallback when the reference library was not built

        perm_in = hs.compute_ordering(pattern)
    return np.argsort(perm_in).astype(np.int32)


def auto_block(nev: int) -> int:
    return 8 if nev >= 32 else (4 if nev >= 8 else (2 if nev >= 3 else 1))


class CpuPencil:
    """A pencil analysed once (ordering + symbolic analysis of the union pattern) with norm estimates."""

    def __init__(self, a, b=None, seed: int = 2026):
        self.a = sp.csr_matrix(a)
        self.n = self.a.shape[0]
        self.b = sp.csr_matrix(b) if b is not None else sp.identity(self.n, format="csr")
        pattern = (abs(self.a) + abs(self.b)).tocsr()
        t0 = time.perf_counter()
        self.fac = OracleLDLT(pattern, order=_ordering(pattern), relax=True)
        self.analyze_s = time.perf_counter() - t0
        rng = np.random.default_rng(seed)
        self.norm_a = float(abs(spla.eigsh(self.a, k=1, which="LM", tol=1e-3, ncv=30,
                                           v0=rng.standard_normal(self.n), return_eigenvectors=False)[0]))
        self.norm_b = 1.0 if b is None else float(abs(spla.eigsh(self.b, k=1, which="LM", tol=1e-3, ncv=30,
                                                                 v0=rng.standard_normal(self.n),
                                                                 return_eigenvectors=False)[0]))
        self.scale = self.norm_a / self.norm_b if self.norm_b > 0 else self.norm_a
        self.factorizations = 0
        self.solve_columns = 0

    def factorize(self, s: float) -> bool:
        self.factorizations += 1
        ok, _, _ = self.fac.factorize((self.a - s * self.b).tocsr())
        self._neg = None
        return ok

    def count_below(self, s: float, direction: float):
        """(nu_-(A - s B), s) with outward moves of a singular endpoint (at most 8)."""
        for t in range(8):
            self.factorizations += 1
            ok, (neg, _, _), _ = self.fac.factorize((self.a - s * self.b).tocsr())
            if ok:
                return neg, s
            s += direction * 1e-7 * (self.scale + abs(s)) * (t + 1)
        raise RuntimeError(f"inertia count singular at every moved endpoint near {s}")

    def op(self, x):
        """(A - sigma B)^{-1} B x for the factorization held."""
        self.solve_columns += x.shape[1]
        return self.fac.solve(self.b @ x)


def _bgram(v, bw):
    return v.T @ bw


def krylov_schur(P: CpuPencil, nev: int, nev_strict: int, p: int, tol: float, seed: int,
                 max_restarts: int = 1000, tol_buffer: float = 1e-8):
    """Wanted (largest |theta|) Ritz pairs of OP = K^{-1} B: (theta, X) with X B-orthonormal."""
    n = P.n
    rng = np.random.default_rng(seed)
    mmax = max(2 * nev + 1, nev + 16) + 4 * p
    mmax = max(mmax, nev + 2 * p)
    mmax = (mmax + p - 1) // p * p
    mmax = min(mmax, n // p * p)
    V = np.zeros((n, mmax + p), order="F")  # column blocks contiguous for the BLAS products
    BV = np.zeros((n, mmax + p), order="F")

    def ortho_block(j):
        """B-orthonormalise V[:, j:j+p] against V[:, :j] (CGS2) and itself (CholQR2): (H, R)."""
        H = np.zeros((j, p))
        for attempt in range(4):
            if attempt:
                V[:, j:j + p] = rng.standard_normal((n, p))
                H[:] = 0.0
            for _ in range(2):
                if j:
                    G = BV[:, :j].T @ V[:, j:j + p]
                    V[:, j:j + p] -= V[:, :j] @ G
                    H += G
            R = np.eye(p)
            ok = True
            for _ in range(2):
                BV[:, j:j + p] = P.b @ V[:, j:j + p]
                G = V[:, j:j + p].T @ BV[:, j:j + p]
                G = 0.5 * (G + G.T)
                try:
                    L = np.linalg.cholesky(G)
                except np.linalg.LinAlgError:
                    ok = False
                    break
                Linv_t = sla.solve_triangular(L, np.eye(p), lower=True).T
                V[:, j:j + p] = V[:, j:j + p] @ Linv_t
                BV[:, j:j + p] = BV[:, j:j + p] @ Linv_t
                R = L.T @ R
            if ok:
                return H, (R if attempt == 0 else np.zeros((p, p)))
        raise RuntimeError("Krylov basis: breakdown")

    V[:, :p] = rng.standard_normal((n, p))
    ortho_block(0)
    tdim = mmax + p
    T = np.zeros((tdim, tdim))
    m = 0
    restarts = 0
    while True:
        while m + p <= mmax:
            j0 = m
            V[:, j0 + p:j0 + 2 * p] = P.op(V[:, j0:j0 + p])
            H, R = ortho_block(j0 + p)
            jh = j0 + p
            T[:jh, j0:j0 + p] = H
            T[j0:j0 + p, :jh] = H.T
            blk = T[j0:j0 + p, j0:j0 + p]
            T[j0:j0 + p, j0:j0 + p] = 0.5 * (blk + blk.T)
            T[jh:jh + p, j0:j0 + p] = R
            T[j0:j0 + p, jh:jh + p] = R.T
            m += p
        w, S = np.linalg.eigh(T[:m, :m])
        rn = np.linalg.norm(T[m:m + p, :m] @ S, axis=0)
        order = sorted(range(m), key=lambda i: -abs(w[i]))
        q0 = 0
        while q0 < m:  # equal Ritz values ranked by residual
            q1 = q0 + 1
            ref = abs(w[order[q0]])
            while q1 < m and abs(w[order[q1]] - w[order[q0]]) <= 1e-12 * ref:
                q1 += 1
            if q1 - q0 > 1:
                order[q0:q1] = sorted(order[q0:q1], key=lambda i: rn[i])
            q0 = q1
        strict = min(nev_strict, nev) if nev_strict > 0 else nev

        def tol_at(q):
            return tol if q < strict else max(tol, tol_buffer)

        nconv = sum(1 for q in range(min(nev, m)) if rn[order[q]] <= tol_at(q) * abs(w[order[q]]))
        if nconv >= min(nev, m) or restarts >= max_restarts:
            take = min(nev, m)
            sel = order[:take]
            conv = [rn[i] <= tol_at(q) * abs(w[i]) for q, i in enumerate(sel)]
            X = V[:, :m] @ S[:, sel]
            return w[sel], X, np.array(conv), restarts
        keep = min(mmax - p, max(nev + p, (nev + mmax) // 2))
        sel = order[:keep]
        Q = S[:, sel]
        th = w[sel]
        Vk = np.asfortranarray(V[:, :m] @ Q)
        BVk = np.asfortranarray(BV[:, :m] @ Q)
        V[:, keep:keep + p] = V[:, m:m + p]
        BV[:, keep:keep + p] = BV[:, m:m + p]
        V[:, :keep] = Vk
        BV[:, :keep] = BVk
        coup = T[m:m + p, :m] @ Q
        Tn = np.zeros_like(T)
        Tn[:keep, :keep] = np.diag(th)
        Tn[keep:keep + p, :keep] = coup
        Tn[:keep, keep:keep + p] = coup.T
        min_wanted = min(abs(w[order[q]]) for q in range(min(nev, m)))
        lock_tol = 4.0 * np.finfo(float).eps * min_wanted
        for q in range(keep):
            if np.linalg.norm(Tn[keep:keep + p, q]) <= lock_tol:
                Tn[keep:keep + p, q] = 0.0
                Tn[q, keep:keep + p] = 0.0
        T = Tn
        m = keep
        restarts += 1


def solve_interval(P: CpuPencil, lower: float, upper: float, tol: float = 1e-10, slice_size: int = 96,
                   seed: int = 2026):
    """Certified interval solve: (eigenvalues ascending, vectors, report dict)."""
    t0 = time.perf_counter()
    nlo, lo = P.count_below(lower, -1.0)
    nhi, hi = P.count_below(upper, +1.0)
    cuts, below = [lo, hi], [nlo, nhi]
    i = 0
    while i + 1 < len(cuts):
        c = below[i + 1] - below[i]
        if c > slice_size and cuts[i + 1] - cuts[i] > 1e-9 * (P.scale + abs(cuts[i])):
            mid = 0.5 * (cuts[i] + cuts[i + 1])
            nm, mid = P.count_below(mid, +1.0)
            cuts.insert(i + 1, mid)
            below.insert(i + 1, nm)
            continue
        i += 1
    lam_all, vec_all, passed = [], [], True
    for i in range(len(cuts) - 1):
        c = below[i + 1] - below[i]
        if c == 0:
            continue
        sigma = 0.5 * (cuts[i] + cuts[i + 1])
        if not P.factorize(sigma):
            raise RuntimeError(f"slice shift singular near {sigma}")
        nev = min(P.n - 1, c + max(4, c // 4))
        p = auto_block(nev)
        for attempt in range(4):
            theta, X, conv, _ = krylov_schur(P, nev, c, p, tol * 0.1, seed + 17 * i + attempt)
            lam = sigma + 1.0 / theta
            inside = [q for q in range(lam.size) if conv[q] and cuts[i] <= lam[q] < cuts[i + 1]]
            if len(inside) == c or attempt == 3:
                break
            nev = min(P.n - 1, nev + max(4, c - len(inside) + 4))
        passed = passed and len(inside) == c
        lam_all.extend(lam[inside])
        vec_all.append(X[:, inside])
    order = np.argsort(lam_all, kind="stable")
    lam = np.asarray(lam_all)[order]
    X = np.hstack(vec_all)[:, order] if vec_all else np.zeros((P.n, 0))
    r = P.a @ X - (P.b @ X) * lam
    eta = np.linalg.norm(r, axis=0) / ((P.norm_a + np.abs(lam) * P.norm_b) * np.linalg.norm(X, axis=0))
    count = nhi - nlo
    success = bool(passed and lam.size == count and np.all(eta <= tol))
    report = {"count_inertia": int(count), "count_found": int(lam.size), "success": success,
              "max_backward_error": float(eta.max()) if eta.size else 0.0,
              "factorizations": P.factorizations, "seconds": time.perf_counter() - t0, "threads": threads()}
    return lam, X, report


def solve_nearest(P: CpuPencil, sigma: float, k: int, tol: float = 1e-10, seed: int = 2026):
    """Certified k nearest to sigma: the window at the first gap after the k-th pair, its ends counted
    (src/driver/definite.cpp:462,700-745)."""
    t0 = time.perf_counter()
    if not P.factorize(sigma):
        raise RuntimeError(f"A - sigma B singular at sigma = {sigma}")
    nev = min(P.n - 1, k + max(4, (k + 1) // 2))
    p = auto_block(nev)
    for attempt in range(4):
        theta, X, conv, _ = krylov_schur(P, nev, k, p, tol * 0.1, seed + attempt)
        lam = sigma + 1.0 / theta
        keep = [q for q in range(lam.size) if conv[q]]
        keep.sort(key=lambda q: abs(lam[q] - sigma))
        d = [abs(lam[q] - sigma) for q in keep]
        gap = next((i + 1 for i in range(k - 1, len(d) - 1)
                    if d[i + 1] - d[i] > 1e-8 * (abs(sigma) + d[i + 1] + P.scale * 1e-3)), None)
        if len(keep) < k or gap is None:
            nev = min(P.n - 1, nev + max(4, nev // 2))
            continue
        R = 0.5 * (d[gap - 1] + d[gap])
        nlo, lo = P.count_below(sigma - R, -1.0)
        nhi, hi = P.count_below(sigma + R, +1.0)
        found = sum(1 for q in keep if lo <= lam[q] < hi)
        if nhi - nlo != found:
            nev = min(P.n - 1, nev + (nhi - nlo - found) + 4)
            if not P.factorize(sigma):
                raise RuntimeError("working shift singular")
            continue
        sel = keep[:k]
        lam_k, X_k = lam[sel], X[:, sel]
        r = P.a @ X_k - (P.b @ X_k) * lam_k
        eta = np.linalg.norm(r, axis=0) / ((P.norm_a + np.abs(lam_k) * P.norm_b) * np.linalg.norm(X_k, axis=0))
        order = np.argsort(lam_k)
        success = bool(np.all(eta <= tol))
        return lam_k[order], X_k[:, order], {"count_inertia": int(nhi - nlo), "count_found": int(found),
                                             "success": success, "max_backward_error": float(eta.max()),
                                             "factorizations": P.factorizations,
                                             "seconds": time.perf_counter() - t0, "threads": threads()}
    raise RuntimeError("nearest target: no certified set after reruns")


def certified_solve(a, b, target: dict, seed: int = 2026):
    """One call of the whole path, as hs::solve runs it: analysis (ordering, symbolic), the shift
    factorizations and counts, the Krylov iteration and the verification. Returns the report."""
    P = CpuPencil(a, b, seed=seed)
    if "lower" in target:
        _, _, rep = solve_interval(P, target["lower"], target["upper"], seed=seed)
    else:
        _, _, rep = solve_nearest(P, target["sigma"], target["k"], seed=seed)
    rep["analyze_s"] = P.analyze_s
    return rep
