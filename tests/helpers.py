"""Shared test matrices (restated from hsolve tests/cpp/support/fixtures.hpp:64-80)."""
import numpy as np
import scipy.sparse as sp


def laplacian_1d(n):
    return sp.diags([-np.ones(n - 1), 2 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1], format="csr")


def laplacian_2d(nx, ny):
    return (sp.kron(sp.identity(ny), laplacian_1d(nx)) + sp.kron(laplacian_1d(ny), sp.identity(nx))).tocsr()


def random_symmetric(n, density, seed):
    rng = np.random.default_rng(seed)
    m = sp.random(n, n, density=density, random_state=rng, data_rvs=lambda k: rng.standard_normal(k))
    m = (m + m.T) * 0.5 + sp.diags(rng.standard_normal(n))
    return m.tocsr()


def random_spd(n, density, seed):
    rng = np.random.default_rng(seed)
    m = sp.random(n, n, density=density, random_state=rng, data_rvs=lambda k: rng.uniform(-1, 1, k))
    m = (m + m.T) * 0.5
    d = np.asarray(abs(m).sum(axis=1)).ravel() + rng.uniform(1, 2, n)
    return (m + sp.diags(d)).tocsr()


def saddle_point(n1, n2, seed):
    """[[H, C^T], [C, 0]]: zero diagonal block forces 2x2 pivots and delayed pivots."""
    rng = np.random.default_rng(seed)
    h = random_spd(n1, 4.0 / n1, seed)
    c = sp.random(n2, n1, density=3.0 / n1, random_state=rng, data_rvs=lambda k: rng.standard_normal(k))
    c = (c + sp.eye(n2, n1)).tocsr()
    return sp.bmat([[h, c.T], [c, None]], format="csr")
