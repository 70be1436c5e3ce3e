"""Lowest-order Nedelec (Whitney edge) elements on a tetrahedral mesh of a box with PEC walls: the
curl-curl stiffness A and the consistent (non-diagonal, SPD) mass B of the Maxwell cavity problem
curl (mu^-1 curl E) = k^2 eps E, tangential E = 0 on the walls.

Mesh. The box [0, Lx] x [0, Ly] x [0, Lz] is cut into nx x ny x nz cells and every cell into six
tetrahedra around its main diagonal (Kuhn / Freudenthal subdivision): tetrahedron p of a cell walks
from the cell's corner (0, 0, 0) to (1, 1, 1) by unit steps along the axes in the order of the p-th
permutation. Every cell uses the same diagonal, so the two cuts of a shared face coincide and the
mesh is conforming. Vertices are numbered v = (i (ny + 1) + j) (nz + 1) + k; along such a walk the
number grows, so a tetrahedron's local vertex order is also its global order.

Unknowns. One per edge that does not lie in a wall (both end points on one wall plane), in the order
of the edge key (lower vertex, higher vertex); an edge is oriented from its lower to its higher
vertex, the orientation of every tetrahedron that contains it.

Basis and element matrices. With barycentric coordinates l_0..l_3, the edge (a, b), a < b, carries
N_ab = l_a grad l_b - l_b grad l_a with curl N_ab = 2 grad l_a x grad l_b, so on a tetrahedron T
  A_T[ab, cd] = |T| / mu  curl N_ab . curl N_cd,
  B_T[ab, cd] = eps (  I_ac g_bd - I_ad g_bc - I_bc g_ad + I_bd g_ac ),
where g_pq = grad l_p . grad l_q and I_pq = int_T l_p l_q = |T| (1 + delta_pq) / 20. All tetrahedra
of one permutation are translates of each other, so the six element matrices are computed once.

Checks that follow from the construction (tests/test_nedelec_gen.py): B is SPD; A is symmetric
positive semi-definite with a null space of dimension (nx - 1)(ny - 1)(nz - 1), the gradients of the
interior vertices' hat functions (the discrete exact sequence on a contractible box); and the
nonzero eigenvalues converge at O(h^2) to the cavity spectrum
  k^2 = pi^2 ((l / Lx)^2 + (m / Ly)^2 + (n / Lz)^2),
l, m, n >= 0 integers with at most one of them zero, twice (TE and TM) when none is zero.

The reference project has no tetrahedral generator (its 3-D inputs are Yee/FIT grids, its Nedelec
elements are 2-D waveguide cross-sections); this one is written from the finite-element definitions
above.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

# local edges of a tetrahedron (local vertex pairs a < b)
_EDGES = ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))
_PERMS = tuple(itertools.permutations(range(3)))


@dataclass(frozen=True)
class TetBox:
    """nx x ny x nz cells of the box [0, Lx] x [0, Ly] x [0, Lz], six tetrahedra per cell, PEC walls."""

    cells: tuple[int, int, int]
    lengths: tuple[float, float, float] = (2.0, 1.0, 0.5)

    def __post_init__(self):
        if len(self.cells) != 3 or min(self.cells) < 1 or min(self.lengths) <= 0:
            raise ValueError("need 3 dimensions, >= 1 cell each, positive lengths")
        object.__setattr__(self, "cells", tuple(int(c) for c in self.cells))
        object.__setattr__(self, "lengths", tuple(float(x) for x in self.lengths))

    @property
    def h(self):
        return tuple(L / N for L, N in zip(self.lengths, self.cells))

    @property
    def n_vertices(self) -> int:
        nx, ny, nz = self.cells
        return (nx + 1) * (ny + 1) * (nz + 1)

    @property
    def n_interior_vertices(self) -> int:
        nx, ny, nz = self.cells
        return (nx - 1) * (ny - 1) * (nz - 1)

    @property
    def n_tetrahedra(self) -> int:
        nx, ny, nz = self.cells
        return 6 * nx * ny * nz


def _element_matrices(h):
    """Stiffness (for mu = 1) and mass (for eps = 1) element matrices of the six Kuhn tetrahedra of a
    cell with edge lengths h, each 6 x 6 over _EDGES."""
    hx, hy, hz = h
    vol = hx * hy * hz / 6.0
    out_a, out_b = [], []
    for perm in _PERMS:
        x = np.zeros((4, 3))
        for s, d in enumerate(perm):
            x[s + 1] = x[s]
            x[s + 1, d] += h[d]
        jac = (x[1:] - x[0]).T                       # columns x_s - x_0
        g = np.empty((4, 3))
        g[1:] = np.linalg.inv(jac)                  # row s-1 of J^-1 = grad l_s
        g[0] = -g[1:].sum(axis=0)
        gg = g @ g.T
        integ = vol * (np.ones((4, 4)) + np.eye(4)) / 20.0
        curls = np.array([2.0 * np.cross(g[a], g[b]) for a, b in _EDGES])
        ae = vol * curls @ curls.T
        be = np.empty((6, 6))
        for i, (a, b) in enumerate(_EDGES):
            for j, (c, d) in enumerate(_EDGES):
                be[i, j] = (integ[a, c] * gg[b, d] - integ[a, d] * gg[b, c]
                            - integ[b, c] * gg[a, d] + integ[b, d] * gg[a, c])
        out_a.append(ae)
        out_b.append(be)
    return np.array(out_a), np.array(out_b)


def _tetrahedra(box: TetBox):
    """(ntet, 4) global vertex numbers, tetrahedra ordered cell-major then by permutation; and the
    permutation index of each."""
    nx, ny, nz = box.cells
    sy, sx = nz + 1, (ny + 1) * (nz + 1)
    step = (sx, sy, 1)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    base = (i * sx + j * sy + k).reshape(-1).astype(np.int64)
    offs = np.zeros((6, 4), dtype=np.int64)
    for p, perm in enumerate(_PERMS):
        for s, d in enumerate(perm):
            offs[p, s + 1] = offs[p, s] + step[d]
    tets = (base[:, None, None] + offs[None, :, :]).reshape(-1, 4)
    pidx = np.tile(np.arange(6), base.size)
    return tets, pidx


def _vertex_coords(box: TetBox, v):
    nx, ny, nz = box.cells
    k = v % (nz + 1)
    j = (v // (nz + 1)) % (ny + 1)
    i = v // ((ny + 1) * (nz + 1))
    return i, j, k


def edges(box: TetBox):
    """(keys, dof, tet_edge): the sorted edge keys lo * nv + hi, the unknown number of every edge
    (-1 for an edge in a wall) and the (ntet, 6) edge numbers of the tetrahedra."""
    tets, _ = _tetrahedra(box)
    nv = box.n_vertices
    lo = np.stack([tets[:, a] for a, _ in _EDGES], axis=1)
    hi = np.stack([tets[:, b] for _, b in _EDGES], axis=1)
    keys, inv = np.unique((lo * nv + hi).reshape(-1), return_inverse=True)
    el, eh = keys // nv, keys % nv
    nx, ny, nz = box.cells
    il, jl, kl = _vertex_coords(box, el)
    ih, jh, kh = _vertex_coords(box, eh)
    wall = np.zeros(keys.size, dtype=bool)
    for cl, ch, top in ((il, ih, nx), (jl, jh, ny), (kl, kh, nz)):
        wall |= ((cl == 0) & (ch == 0)) | ((cl == top) & (ch == top))
    dof = np.full(keys.size, -1, dtype=np.int64)
    dof[~wall] = np.arange(int((~wall).sum()))
    return keys, dof, inv.reshape(-1, 6)


def _cell_values(box: TetBox, value, centroids):
    if callable(value):
        return np.asarray(value(centroids), dtype=np.float64).reshape(-1)
    return np.full(centroids.shape[0], float(value))


def assemble(box: TetBox, eps=1.0, mu=1.0):
    """(A, B): curl-curl stiffness and consistent mass on the interior edges, CSR float64. eps and mu
    are constants or callables of the (ntet, 3) tetrahedron centroids."""
    tets, pidx = _tetrahedra(box)
    ae, be = _element_matrices(box.h)
    _, dof, te = edges(box)
    need_centroids = callable(eps) or callable(mu)
    if need_centroids:
        h = np.array(box.h)
        i, j, k = _vertex_coords(box, tets)
        xyz = np.stack([i, j, k], axis=-1) * h
        cen = xyz.mean(axis=1)
    else:
        cen = np.zeros((tets.shape[0], 3))
    e_t = _cell_values(box, eps, cen)
    nu_t = 1.0 / _cell_values(box, mu, cen)
    d = dof[te]                                       # (ntet, 6)
    rows = np.repeat(d, 6, axis=1).reshape(-1)
    cols = np.tile(d, (1, 6)).reshape(-1)
    keep = (rows >= 0) & (cols >= 0)
    av = (ae[pidx] * nu_t[:, None, None]).reshape(-1)
    bv = (be[pidx] * e_t[:, None, None]).reshape(-1)
    n = int(dof.max()) + 1 if dof.size and dof.max() >= 0 else 0
    a = sp.csr_matrix((av[keep], (rows[keep], cols[keep])), shape=(n, n))
    b = sp.csr_matrix((bv[keep], (rows[keep], cols[keep])), shape=(n, n))
    for m in (a, b):
        m.sum_duplicates()
        m.sort_indices()
    # exact symmetry: the element matrices are symmetric up to rounding in the products above
    a = ((a + a.T) * 0.5).tocsr()
    b = ((b + b.T) * 0.5).tocsr()
    a.sort_indices()
    b.sort_indices()
    return a, b


def pencil(box: TetBox, eps=1.0, mu=1.0):
    """The generalized pencil (A, B) of the cavity (B is not diagonal: there is no standard form)."""
    return assemble(box, eps, mu)


def cavity_eigenvalues(lengths, kmax2: float):
    """Sorted k^2 <= kmax2 of the PEC box (continuous problem), with multiplicity."""
    lx, ly, lz = lengths
    out = []
    lim = [int(np.sqrt(kmax2) * L / np.pi) + 1 for L in (lx, ly, lz)]
    for l in range(lim[0] + 1):
        for m in range(lim[1] + 1):
            for n in range(lim[2] + 1):
                zeros = (l == 0) + (m == 0) + (n == 0)
                if zeros > 1:
                    continue
                k2 = np.pi ** 2 * ((l / lx) ** 2 + (m / ly) ** 2 + (n / lz) ** 2)
                if k2 <= kmax2:
                    out.extend([k2] * (2 if zeros == 0 else 1))
    return np.sort(np.array(out))


# PEC box 2 x 1 x 0.5 (the benchmark box of Nedelec-tetrahedron meshes), by size
BOX_2x1x05_SMALL = TetBox((12, 6, 3))          # n = 1,155
BOX_2x1x05_1E5 = TetBox((50, 25, 13))          # n = 107,163
BOX_2x1x05_1E6 = TetBox((106, 53, 27))         # n = 1,032,255
