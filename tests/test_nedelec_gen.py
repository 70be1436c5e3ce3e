"""CPU: the Nedelec-tetrahedron cavity generator (hsolve_b200.gen.nedelec) checked against what the
discretization must satisfy, and its pencils through the oracle's inertia.

There is no closed-form discrete spectrum for these meshes, so the checks are: B symmetric positive
definite; A symmetric positive semi-definite with exactly (nx-1)(ny-1)(nz-1) zero eigenvalues (the
gradients of interior vertex functions); the nonzero eigenvalues converging at O(h^2) to the PEC
cavity spectrum; and the oracle's Sylvester counts of A - sigma B equal to dense counts.
"""
import numpy as np
import pytest
import scipy.linalg as sl
import scipy.sparse.linalg as sla

from hsolve_b200.gen import nedelec as ne
from oracle.ldlt import OracleLDLT


@pytest.mark.parametrize("cells", [(2, 2, 2), (4, 2, 2), (3, 3, 2), (5, 3, 2)])
def test_null_space_and_definiteness(cells):
    box = ne.TetBox(cells, (2.0, 1.0, 0.5))
    a, b = ne.assemble(box)
    A, B = a.toarray(), b.toarray()
    assert np.array_equal(A, A.T) and np.array_equal(B, B.T)
    assert np.linalg.eigvalsh(B).min() > 0
    w = sl.eigh(A, B, eigvals_only=True)
    tol = 1e-9 * w.max()
    assert w.min() > -tol
    assert int(np.count_nonzero(np.abs(w) < tol)) == box.n_interior_vertices


def test_eigenvalues_converge_to_the_cavity():
    exact = ne.cavity_eigenvalues((2.0, 1.0, 0.5), 45.0)[:5]   # 12.34, 19.74, 32.08, 41.95, 41.95
    errs = []
    for cells in [(12, 6, 3), (24, 12, 6)]:
        a, b = ne.assemble(ne.TetBox(cells))
        w = np.sort(sla.eigsh(a, k=6, M=b, sigma=25.0, which="LM", return_eigenvectors=False))[:5]
        errs.append(np.abs(w - exact) / exact)
    assert np.all(errs[1] < 0.01)
    assert np.all(errs[0] / errs[1] > 3.0)            # O(h^2): halving h divides the error by ~4


def test_cavity_spectrum_multiplicities():
    ex = ne.cavity_eigenvalues((1.0, 1.0, 1.0), 3.0 * np.pi ** 2 + 1e-9)
    # (1,1,0)x3 at 2 pi^2 (one zero each), (1,1,1) at 3 pi^2 twice (TE + TM)
    assert np.allclose(ex, [2 * np.pi ** 2] * 3 + [3 * np.pi ** 2] * 2)


@pytest.mark.parametrize("sigma", [10.0, 25.0, 45.0])
def test_oracle_inertia_matches_dense(sigma):
    box = ne.TetBox((8, 4, 2))
    a, b = ne.assemble(box)
    w = sl.eigh(a.toarray(), b.toarray(), eigvals_only=True)
    assert np.min(np.abs(w - sigma)) > 1e-6 * sigma    # sigma is not an eigenvalue
    k = (a - sigma * b).tocsr()
    valid, (neg, zero, pos), _ = OracleLDLT(k).factorize(k)
    assert valid and zero == 0
    assert neg == int(np.count_nonzero(w < sigma))
    assert neg + pos == a.shape[0]


def test_presets_and_materials():
    for box, n in [(ne.BOX_2x1x05_SMALL, 1155), (ne.BOX_2x1x05_1E5, 107163), (ne.BOX_2x1x05_1E6, 1032255)]:
        _, dof, _ = ne.edges(box)
        assert int(np.count_nonzero(dof >= 0)) == n
    box = ne.TetBox((3, 2, 2))
    a1, b1 = ne.assemble(box)
    a2, b2 = ne.assemble(box, eps=lambda c: np.full(c.shape[0], 4.0), mu=2.0)
    np.testing.assert_allclose(b2.toarray(), 4.0 * b1.toarray(), rtol=1e-15, atol=0)
    np.testing.assert_allclose(a2.toarray(), 0.5 * a1.toarray(), rtol=1e-15, atol=0)
