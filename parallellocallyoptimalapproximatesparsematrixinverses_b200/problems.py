"""Seeded synthetic SPD operators for the benchmark workloads (numpy PCG64
generators, `numpy.random.default_rng(seed)`).

* laplacian_2d(m): 5-point Laplacian on an m x m grid, Dirichlet boundary,
  diagonal 4, off-diagonals -1 (m = 64: n = 4096, nnz = 20,224).
* diffusion_3d(m, sigma, seed): 7-point variable-coefficient diffusion on an
  m^3 grid.  Face coefficients k_f = exp(sigma * xi), xi ~ N(0, 1), drawn for
  the x faces, then the y faces, then the z faces, each block in lexicographic
  order (x fastest); boundary faces add k_f to the diagonal (Dirichlet), so A
  is SPD (m = 64: n = 262,144, nnz = 1,810,432).
* diffusion_2d(m, sigma, seed): the 5-point analogue on an m x m grid.
* random_banded_spd(n, half_width, extra, seed): band of the given half width
  plus `extra` uniformly random off-diagonals per row, pattern symmetrised by
  mirroring the upper triangle; off-diagonals ~ N(0, 1); diagonal = 1.05 x the
  absolute row sum.
* tridiagonal(n): tridiag(-1, 2, -1), the reference's C++ test fixture
  (tests/test.cpp:13-28).
* diffusion_batch(count, seed, n_min, n_max): many independent systems for
  batched runs.  Per system: n log-uniform in [n_min, n_max], a 5-point 2-D
  or 7-point 3-D grid (fair coin) with side round(n^(1/2)) or round(n^(1/3)),
  log-normal coefficients with sigma 0.5, plus a diagonal shift U(0, 0.1).
"""
from __future__ import annotations

import numpy as np
from scipy import sparse


def tridiagonal(n: int) -> sparse.csc_matrix:
    main = np.full(n, 2.0)
    off = np.full(n - 1, -1.0)
    return sparse.diags([off, main, off], [-1, 0, 1], format="csc", dtype=np.float64)


def laplacian_2d(m: int) -> sparse.csc_matrix:
    t = sparse.diags([np.full(m - 1, -1.0), np.full(m, 4.0), np.full(m - 1, -1.0)], [-1, 0, 1], dtype=np.float64)
    s = sparse.diags([np.full(m - 1, -1.0), np.full(m - 1, -1.0)], [-1, 1], dtype=np.float64)
    a = sparse.kron(sparse.identity(m, dtype=np.float64), t) + sparse.kron(s, sparse.identity(m, dtype=np.float64))
    a = sparse.csc_matrix(a)
    a.sum_duplicates()
    a.sort_indices()
    return a


def _assemble(n, rows, cols, vals, diag):
    r = np.concatenate([rows, cols, np.arange(n)])
    c = np.concatenate([cols, rows, np.arange(n)])
    v = np.concatenate([-vals, -vals, diag])
    a = sparse.csc_matrix((v, (r, c)), shape=(n, n), dtype=np.float64)
    a.sum_duplicates()
    a.sort_indices()
    return a


def diffusion_3d(m: int, sigma: float = 1.0, seed: int = 0) -> sparse.csc_matrix:
    rng = np.random.default_rng(seed)
    n = m ** 3
    # face coefficients: axis-x faces have shape (m, m, m+1) indexed [k, j, i_face], etc.
    kx = np.exp(sigma * rng.standard_normal((m, m, m + 1)))
    ky = np.exp(sigma * rng.standard_normal((m, m + 1, m)))
    kz = np.exp(sigma * rng.standard_normal((m + 1, m, m)))
    idx = np.arange(n).reshape(m, m, m)  # [k, j, i], index = i + m*j + m*m*k
    diag = np.zeros((m, m, m))
    diag += kx[:, :, :-1] + kx[:, :, 1:]
    diag += ky[:, :-1, :] + ky[:, 1:, :]
    diag += kz[:-1, :, :] + kz[1:, :, :]
    rows = [idx[:, :, :-1].ravel(), idx[:, :-1, :].ravel(), idx[:-1, :, :].ravel()]
    cols = [idx[:, :, 1:].ravel(), idx[:, 1:, :].ravel(), idx[1:, :, :].ravel()]
    vals = [kx[:, :, 1:-1].ravel(), ky[:, 1:-1, :].ravel(), kz[1:-1, :, :].ravel()]
    return _assemble(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals), diag.ravel())


def diffusion_2d(m: int, sigma: float = 1.0, seed: int = 0) -> sparse.csc_matrix:
    rng = np.random.default_rng(seed)
    n = m * m
    kx = np.exp(sigma * rng.standard_normal((m, m + 1)))
    ky = np.exp(sigma * rng.standard_normal((m + 1, m)))
    idx = np.arange(n).reshape(m, m)  # [j, i]
    diag = kx[:, :-1] + kx[:, 1:] + ky[:-1, :] + ky[1:, :]
    rows = [idx[:, :-1].ravel(), idx[:-1, :].ravel()]
    cols = [idx[:, 1:].ravel(), idx[1:, :].ravel()]
    vals = [kx[:, 1:-1].ravel(), ky[1:-1, :].ravel()]
    return _assemble(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals), diag.ravel())


def random_banded_spd(n: int, half_width: int = 4, extra: int = 6, seed: int = 0) -> sparse.csc_matrix:
    rng = np.random.default_rng(seed)
    rows = []
    cols = []
    for d in range(1, half_width + 1):
        r = np.arange(n - d)
        rows.append(r)
        cols.append(r + d)
    r = np.repeat(np.arange(n), extra)
    c = rng.integers(0, n, size=r.size)
    keep = r != c
    rows.append(np.minimum(r[keep], c[keep]))
    cols.append(np.maximum(r[keep], c[keep]))
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    upper = sparse.coo_matrix((np.ones(rows.size), (rows, cols)), shape=(n, n)).tocsr()
    upper.sum_duplicates()
    upper = upper.tocoo()
    vals = rng.standard_normal(upper.nnz)
    off = sparse.coo_matrix((vals, (upper.row, upper.col)), shape=(n, n))
    sym = (off + off.T).tocsr()
    diag = 1.05 * np.asarray(abs(sym).sum(axis=1)).ravel()
    diag[diag == 0.0] = 1.0
    a = sparse.csc_matrix(sym + sparse.diags(diag))
    a.sum_duplicates()
    a.sort_indices()
    return a


def diffusion_batch(count: int = 256, seed: int = 0, n_min: int = 1000, n_max: int = 64000):
    rng = np.random.default_rng(seed)
    out = []
    for b in range(count):
        n = float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        three_d = bool(rng.integers(0, 2))
        system_seed = int(rng.integers(0, 2**31 - 1))
        shift = float(rng.uniform(0.0, 0.1))
        if three_d:
            a = diffusion_3d(max(2, int(round(n ** (1.0 / 3.0)))), 0.5, system_seed)
        else:
            a = diffusion_2d(max(2, int(round(n ** 0.5))), 0.5, system_seed)
        a = sparse.csc_matrix(a + shift * sparse.identity(a.shape[0], format="csc"))
        a.sum_duplicates()
        a.sort_indices()
        out.append(a)
    return out


def diagonal_inverse(a) -> sparse.csc_matrix:
    """diag(A)^-1 as a sparse diagonal (the reference's default Pr, methods_common.cpp:50-63)."""
    d = a.diagonal()
    return sparse.diags(1.0 / d, format="csc", dtype=np.float64)


def solution_rhs(a, seed: int = 0):
    """x* ~ N(0, 1) with default_rng(seed) and b = A x*."""
    x = np.random.default_rng(seed).standard_normal(a.shape[0])
    return a @ x, x
