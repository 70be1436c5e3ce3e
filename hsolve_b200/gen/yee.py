"""Yee / finite-integration (FIT) curl-curl pencils on a box: the synthetic inputs of the benchmarks.

Same discretization, unknown layout and material rules as the reference generator
(tools/gen/yee.py:1-34 in hsolve), built here from explicit index arithmetic:

* unknowns are line integrals u_e = h_e E_e on primal edges, ordered x-edges, y-edges, z-edges,
  each block in C order over (x, y, z) of (cell, node, node) / (node, cell, node) /
  (node, node, cell); a PEC wall removes the edges lying in it, a Bloch-periodic box keeps all
  3 Nx Ny Nz edges and multiplies couplings that wrap around by exp(i phase_d);
* faces are ordered x-, y-, z-faces over (node, cell, cell) / (cell, node, cell) /
  (cell, cell, node) and (C u)_x = d_y u_z - d_z u_y (cyclic);
* A = C^H diag(nu_f |f~|/|f|) C (Hermitian part), B = diag(eps_e |e~|/|e|) with eps averaged over
  the 4 cells around an edge and 1/mu over the 2 cells a face separates;
* the standard form is B^{-1/2} A B^{-1/2}.

The unknown ordering and the assembly formula must match the reference's so that the same
(sigma, k) targets and the same exact spectra apply (reference: tools/gen/yee.py:151-208).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp


@dataclass(frozen=True)
class Box:
    """cells[d] cells over length lengths[d]; boundary 'pec' or 'bloch' with phases[d] = k_d L_d."""

    cells: tuple[int, int, int]
    lengths: tuple[float, float, float] = (1.0, 1.0, 1.0)
    boundary: str = "pec"
    phases: tuple[float, float, float] = (0.0, 0.0, 0.0)

    def __post_init__(self):
        if self.boundary not in ("pec", "bloch"):
            raise ValueError("boundary must be 'pec' or 'bloch'")
        lo = 2 if self.boundary == "pec" else 1
        if len(self.cells) != 3 or min(self.cells) < lo or min(self.lengths) <= 0:
            raise ValueError("need 3 dimensions, >= 2 cells (PEC) / >= 1 (Bloch), positive lengths")
        if self.boundary == "pec" and any(p != 0.0 for p in self.phases):
            raise ValueError("phases need boundary='bloch'")
        object.__setattr__(self, "cells", tuple(int(c) for c in self.cells))
        object.__setattr__(self, "lengths", tuple(float(x) for x in self.lengths))
        object.__setattr__(self, "phases", tuple(_phase_mod(p) for p in self.phases))

    @property
    def h(self):
        return tuple(L / N for L, N in zip(self.lengths, self.cells))

    def nodes(self, d):
        return self.cells[d] - 1 if self.boundary == "pec" else self.cells[d]

    @property
    def n_edges(self):
        c = self.cells
        nd = [self.nodes(d) for d in range(3)]
        return c[0] * nd[1] * nd[2] + nd[0] * c[1] * nd[2] + nd[0] * nd[1] * c[2]

    @property
    def complex(self):
        return any(not _is_real_phase(p) for p in self.phases)

    def null_dim(self):
        nn = self.nodes(0) * self.nodes(1) * self.nodes(2)
        if self.boundary == "pec":
            return nn
        return nn + (2 if all(p == 0.0 for p in self.phases) else 0)


def _phase_mod(p):
    q = float(np.mod(p, 2 * np.pi))
    return 0.0 if q >= 2 * np.pi else q


def _is_real_phase(p):
    r = p / np.pi
    return r == round(r)


def _wrap(p):
    r = p / np.pi
    if r == round(r):
        return 1.0 if int(round(r)) % 2 == 0 else -1.0
    return complex(np.exp(1j * p))


def _diff_entries(box: Box, d: int):
    """1-D difference (cells x nodes along d): list of (cell, node, value) triples."""
    n = box.cells[d]
    if box.boundary == "pec":
        # cell c spans nodes c and c+1 of the full line; interior node q <-> full node q+1
        cells, nodes, vals = [], [], []
        for c in range(n):
            if c + 1 <= n - 1:  # right node c+1 is interior -> +1
                cells.append(c), nodes.append(c), vals.append(1.0)
            if c >= 1:  # left node c is interior -> -1
                cells.append(c), nodes.append(c - 1), vals.append(-1.0)
        return np.array(cells), np.array(nodes), np.array(vals, dtype=float)
    w = _wrap(box.phases[d])
    c = np.arange(n)
    cells = np.concatenate((c, c))
    nodes = np.concatenate((c, (c + 1) % n))
    vals = np.concatenate((-np.ones(n), np.ones(n))).astype(complex if box.complex else float)
    vals[2 * n - 1] = w  # the last cell reaches node 0 across the period
    return cells, nodes, vals


def _block_index(shape, i, j, k):
    return (np.asarray(i) * shape[1] + np.asarray(j)) * shape[2] + np.asarray(k)


def curl(box: Box) -> sp.csr_matrix:
    """Topological curl (faces x edges)."""
    N = box.cells
    nd = tuple(box.nodes(d) for d in range(3))
    edge_shape = [(N[0], nd[1], nd[2]), (nd[0], N[1], nd[2]), (nd[0], nd[1], N[2])]
    face_shape = [(nd[0], N[1], N[2]), (N[0], nd[1], N[2]), (N[0], N[1], nd[2])]
    e_off = np.cumsum([0] + [int(np.prod(s)) for s in edge_shape])
    f_off = np.cumsum([0] + [int(np.prod(s)) for s in face_shape])
    diffs = [_diff_entries(box, d) for d in range(3)]
    rows, cols, vals = [], [], []

    def add(face_blk, edge_blk, d, sign):
        """Face block face_blk gets sign * D_d applied to edge block edge_blk (identity elsewhere).

        Along dimension d the face index is a cell and the edge index a node; along the other two
        dimensions face and edge share the same (node or cell) index."""
        fs, es = face_shape[face_blk], edge_shape[edge_blk]
        dc, dn, dv = diffs[d]
        other = [a for a in range(3) if a != d]
        g = [np.arange(fs[a]) for a in other]
        o0, o1 = np.meshgrid(g[0], g[1], indexing="ij")
        o0, o1 = o0.ravel(), o1.ravel()
        for c, q, v in zip(dc, dn, dv):
            fi = [None] * 3
            ei = [None] * 3
            fi[d], ei[d] = np.full(o0.size, c), np.full(o0.size, q)
            fi[other[0]], fi[other[1]] = o0, o1
            ei[other[0]], ei[other[1]] = o0, o1
            rows.append(f_off[face_blk] + _block_index(fs, *fi))
            cols.append(e_off[edge_blk] + _block_index(es, *ei))
            vals.append(np.full(o0.size, sign * v))

    # (C u)_x = d_y u_z - d_z u_y ; (C u)_y = d_z u_x - d_x u_z ; (C u)_z = d_x u_y - d_y u_x
    add(0, 2, 1, +1.0), add(0, 1, 2, -1.0)
    add(1, 0, 2, +1.0), add(1, 2, 0, -1.0)
    add(2, 1, 0, +1.0), add(2, 0, 1, -1.0)
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = np.concatenate(vals)
    return sp.csr_matrix((v, (r, c)), shape=(int(f_off[-1]), int(e_off[-1])))


def _avg_weights(box: Box, d: int):
    """Node-along-d averaging of the two adjacent cells: (node, cell, 0.5) triples."""
    n = box.cells[d]
    if box.boundary == "pec":
        q = np.arange(n - 1)  # interior node q sits between cells q and q+1
        return np.concatenate((q, q)), np.concatenate((q, q + 1))
    q = np.arange(n)
    return np.concatenate((q, q)), np.concatenate((q, (q - 1) % n))


def _average_field(box: Box, field, node_dims):
    """Average a cell field onto the index grid where dims in node_dims are nodes (others cells)."""
    out = np.asarray(field, dtype=float)
    for d in node_dims:
        nodes, cells = _avg_weights(box, d)
        nn = box.nodes(d)
        moved = np.moveaxis(out, d, 0)
        acc = np.zeros((nn,) + moved.shape[1:])
        np.add.at(acc, nodes, 0.5 * moved[cells])
        out = np.moveaxis(acc, 0, d)
    return out.ravel()


def _cell_values(box: Box, value):
    if np.ndim(value) == 0:
        if float(value) <= 0:
            raise ValueError("material parameters must be positive")
        return float(value)
    arr = np.asarray(value, dtype=float)
    if arr.shape != box.cells or arr.min() <= 0:
        raise ValueError("cell material array must have shape cells and be positive")
    return arr


def assemble(box: Box, eps=1.0, mu=1.0):
    """FIT pencil (A, B): A = C^H M_nu C (Hermitian part), B = M_eps (diagonal)."""
    hx, hy, hz = box.h
    N = box.cells
    nd = tuple(box.nodes(d) for d in range(3))
    e_sizes = [N[0] * nd[1] * nd[2], nd[0] * N[1] * nd[2], nd[0] * nd[1] * N[2]]
    f_sizes = [nd[0] * N[1] * N[2], N[0] * nd[1] * N[2], N[0] * N[1] * nd[2]]
    eps_c = _cell_values(box, eps)
    nu_c = 1.0 / _cell_values(box, mu) if np.ndim(mu) else 1.0 / _cell_values(box, mu)
    # edges along d: nodes in the other two dims; faces normal to d: node along d only
    if isinstance(eps_c, float):
        eps_e = [np.full(s, eps_c) for s in e_sizes]
    else:
        eps_e = [_average_field(box, eps_c, [a for a in range(3) if a != d]) for d in range(3)]
    if isinstance(nu_c, float):
        nu_f = [np.full(s, nu_c) for s in f_sizes]
    else:
        nu_f = [_average_field(box, nu_c, [d]) for d in range(3)]
    eg = (hy * hz / hx, hx * hz / hy, hx * hy / hz)
    fg = (hx / (hy * hz), hy / (hx * hz), hz / (hx * hy))
    m_eps = np.concatenate([e * g for e, g in zip(eps_e, eg)])
    m_nu = np.concatenate([v * g for v, g in zip(nu_f, fg)])
    c = curl(box)
    a = (c.conj().T @ sp.diags(m_nu) @ c).tocsr()
    a = hermitian_part(a)
    return a, sp.diags(m_eps, format="csr")


def hermitian_part(m) -> sp.csr_matrix:
    """(M + M^H) / 2 with canonical CSR (sorted, summed duplicates)."""
    h = ((m + m.conj().T) * 0.5).tocsr()
    h.sum_duplicates()
    h.sort_indices()
    return h


def standard_form(a, b) -> sp.csr_matrix:
    s = sp.diags(1.0 / np.sqrt(b.diagonal().real))
    return hermitian_part(s @ a @ s)


def pencil(box: Box, form: str = "standard", eps=1.0, mu=1.0):
    """(A, B) of the box: B is None for the standard form (HEP)."""
    a, b = assemble(box, eps, mu)
    if form == "standard":
        return standard_form(a, b), None
    if form == "generalized":
        return a, b
    raise ValueError("form must be 'standard' or 'generalized'")


def sphere_permittivity(box: Box, radius: float, eps_in: float, eps_out: float = 1.0,
                        samples: int = 3) -> np.ndarray:
    """Cell permittivity of a centred dielectric sphere of radius radius*min(L) (volume fraction
    sampled on samples^3 sub-points per cell); the photonic-crystal unit cell."""
    h = box.h
    axes = [((np.arange(n * samples) + 0.5) / samples) * hd - L / 2
            for n, hd, L in zip(box.cells, h, box.lengths)]
    x, y, z = np.meshgrid(*axes, indexing="ij", sparse=True)
    inside = x ** 2 + y ** 2 + z ** 2 <= (radius * min(box.lengths)) ** 2
    nx, ny, nz = box.cells
    frac = inside.reshape(nx, samples, ny, samples, nz, samples).mean(axis=(1, 3, 5))
    return eps_out + (eps_in - eps_out) * frac


# Named boxes of the benchmark workloads (sizes as in the reference presets, tools/gen/yee.py:353-384)
CUBE20 = Box((20, 20, 20))                                  # n = 21,660  (PEC cube 20^3)
BOX_1E4 = Box((20, 16, 12), (1.0, 0.7, 0.45))               # n = 10,228
BOX_1E5 = Box((44, 34, 26), (1.0, 0.75, 0.55))              # n = 109,744
BOX_1E6 = Box((92, 71, 54), (1.0, 0.75, 0.55))              # n = 1,027,733
