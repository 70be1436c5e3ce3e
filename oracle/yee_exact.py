"""ORACLE (test infrastructure only; never imported by the product path).

Closed-form discrete spectrum of the homogeneous Yee/FIT curl-curl pencil on a box, restated from
the formula documented in hsolve's generator (tools/gen/yee.py:20-29, exact_eigenvalues at
tools/gen/yee.py:231-257):

* PEC box:   lambda = (1/(eps mu)) sum_d (2/h_d sin(m_d pi / (2 N_d)))^2, m_d = 0..N_d-1, with two
  polarizations when all three m_d >= 1, one when exactly one m_d = 0, none otherwise; plus the
  gradient null space of dimension prod_d (N_d - 1).
* Bloch box: q_d = phase_d / N_d + 2 pi m_d / N_d (argument phase_d/(2N_d) + m_d pi / N_d),
  two modes per wavevector with a nonzero sum, plus one zero per wavevector (its gradient), and
  the two extra constant fields at k = 0.

The three per-dimension terms are summed in ascending order so permuted index triples give
bitwise-equal values (exact multiplicities). Pinned against the reference's own function by
tests/golden/yee_spectra.npz (generated by tests/golden/make_golden.py).
"""
from __future__ import annotations

import numpy as np


def exact_spectrum(cells, lengths=(1.0, 1.0, 1.0), boundary="pec", phases=(0.0, 0.0, 0.0),
                   eps=1.0, mu=1.0) -> np.ndarray:
    cells = tuple(int(c) for c in cells)
    h = [L / N for L, N in zip(lengths, cells)]
    per_dim = []
    for d in range(3):
        m = np.arange(cells[d], dtype=float)
        if boundary == "pec":
            theta = m * np.pi / (2 * cells[d])
        else:
            theta = phases[d] / (2 * cells[d]) + m * np.pi / cells[d]
        per_dim.append((2.0 / h[d] * np.sin(theta)) ** 2)
    gx, gy, gz = np.meshgrid(per_dim[0], per_dim[1], per_dim[2], indexing="ij")
    trip = np.sort(np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1), axis=1)
    total = (trip[:, 0] + trip[:, 1]) + trip[:, 2]
    if boundary == "pec":
        nonzero = (np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1) > 0).sum(axis=1)
        mult = np.select([nonzero == 3, nonzero == 2], [2, 1], 0)
        null = (cells[0] - 1) * (cells[1] - 1) * (cells[2] - 1)
    else:
        mult = np.where(total > 0, 2, 0)
        null = cells[0] * cells[1] * cells[2]
        if all(p == 0.0 for p in phases):
            null += 2
    w = np.concatenate((np.repeat(total, mult), np.zeros(null)))
    return np.sort(w / (eps * mu))


def count_below(w: np.ndarray, s: float) -> int:
    """Number of eigenvalues strictly below s (the Sylvester count nu_-(A - s B))."""
    return int(np.searchsorted(np.sort(w), s, side="left"))


def mid_gap_shifts(w: np.ndarray, count: int, min_gap: float) -> list[float]:
    """`count` shifts at midpoints of spectral gaps spread over the spectrum (gaps narrower than
    min_gap skipped); the placement rule of hsolve tests/cpp/test_factor.cpp:46-60."""
    w = np.sort(np.asarray(w, dtype=float))
    n = w.size
    out = []
    for t in range(1, count + 1):
        for k in range(n * t // (count + 1), n):
            if k > 0 and w[k] - w[k - 1] > min_gap:
                out.append(0.5 * (w[k - 1] + w[k]))
                break
    return out


def laplacian_1d_spectrum(n: int) -> np.ndarray:
    """tridiag(-1, 2, -1): 2 - 2 cos(k pi/(n+1)), k = 1..n (tests/cpp/support/fixtures.hpp:76-80)."""
    k = np.arange(1, n + 1)
    return np.sort(2.0 - 2.0 * np.cos(k * np.pi / (n + 1)))


def laplacian_2d_spectrum(nx: int, ny: int) -> np.ndarray:
    a = laplacian_1d_spectrum(nx)
    b = laplacian_1d_spectrum(ny)
    return np.sort((a[:, None] + b[None, :]).ravel())
