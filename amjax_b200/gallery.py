"""Sparse model problems used by the tests and the benchmark (host, scipy CSR).

These generators stand in for ``pyamg.gallery`` (the reference builds its test and
benchmark matrices with ``pyamg.gallery.poisson``, tests/test_multilevel.py:7 and
benchmarks/benchmark.ipynb cell 10), which is not importable here.  Every matrix is
returned as a canonical scipy CSR matrix (sorted indices, no duplicates, float64).

Grid ordering is lexicographic with the LAST axis fastest, i.e. the unknown of grid
point (i, j) on an ``(nx, ny)`` grid is ``i * ny + j``.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

__all__ = [
    "poisson",
    "tridiag",
    "anisotropic_diffusion_2d",
    "variable_diffusion_2d",
    "variable_diffusion_3d",
    "convection_diffusion_2d",
]


def _canonical(A) -> sp.csr_matrix:
    A = sp.csr_matrix(A, dtype=np.float64)
    A.sum_duplicates()
    A.eliminate_zeros()
    A.sort_indices()
    return A


def tridiag(n: int, diag: float = 2.0, off: float = -1.0) -> sp.csr_matrix:
    """tridiag(off, diag, off) of size n (the 1-D Dirichlet Laplacian by default)."""
    e = np.ones(n)
    return _canonical(sp.diags([off * e[1:], diag * e, off * e[1:]], [-1, 0, 1], shape=(n, n)))


def poisson(grid, format: str = "csr") -> sp.csr_matrix:
    """Second-order finite-difference Dirichlet Laplacian on a 1-D/2-D/3-D grid.

    The stencil is the (2d+1)-point one with ``2*d`` on the diagonal and ``-1`` for each
    neighbour, the same operator as ``pyamg.gallery.poisson(grid)``.
    """
    del format
    grid = tuple(int(g) for g in grid)
    mats = [tridiag(g) for g in grid]
    eyes = [sp.identity(g, format="csr") for g in grid]
    A = None
    for axis in range(len(grid)):
        term = None
        for d in range(len(grid)):
            f = mats[d] if d == axis else eyes[d]
            term = f if term is None else sp.kron(term, f, format="csr")
        A = term if A is None else A + term
    return _canonical(A)


def _assemble(n_unknowns, rows, cols, vals):
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n_unknowns, n_unknowns))
    return _canonical(A.tocsr())


def anisotropic_diffusion_2d(n: int, epsilon: float, theta: float = np.pi / 4) -> sp.csr_matrix:
    """Rotated anisotropic diffusion ``-div(K grad u)`` on an n x n grid, Dirichlet.

    ``K = Q diag(1, epsilon) Q^T`` with Q the rotation by ``theta``.  Discretised with
    the standard 9-point finite-difference stencil (h = 1): centre ``2a + 2c``,
    east/west ``-a``, north/south ``-c``, NE/SW corners ``-b/2`` and NW/SE corners
    ``+b/2`` with ``a = K_xx, c = K_yy, b = K_xy``.
    """
    cs, sn = np.cos(theta), np.sin(theta)
    a = cs * cs + epsilon * sn * sn
    c = sn * sn + epsilon * cs * cs
    b = (1.0 - epsilon) * cs * sn
    stencil = {(0, 0): 2 * a + 2 * c, (-1, 0): -a, (1, 0): -a, (0, -1): -c, (0, 1): -c,
               (1, 1): -b / 2, (-1, -1): -b / 2, (1, -1): b / 2, (-1, 1): b / 2}
    I, J = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    I = I.ravel(); J = J.ravel()
    rows, cols, vals = [], [], []
    for (di, dj), v in stencil.items():
        if v == 0.0:
            continue
        ii, jj = I + di, J + dj
        ok = (ii >= 0) & (ii < n) & (jj >= 0) & (jj < n)
        rows.append((I * n + J)[ok]); cols.append((ii * n + jj)[ok]); vals.append(np.full(ok.sum(), v))
    return _assemble(n * n, rows, cols, vals)


def _harmonic(a, b):
    return 2.0 * a * b / (a + b)


def _cell_diffusion(shape, kappa):
    """Cell-centred finite-volume ``-div(kappa grad u)`` with harmonic face means.

    Interior faces carry the harmonic mean of the two adjacent cells' kappa; a Dirichlet
    boundary face carries ``2 * kappa_cell`` (the cell centre is h/2 from the wall).
    """
    shape = tuple(shape)
    N = int(np.prod(shape))
    idx = np.arange(N).reshape(shape)
    diag = np.zeros(shape)
    rows, cols, vals = [], [], []
    for ax in range(len(shape)):
        lo = [slice(None)] * len(shape); hi = [slice(None)] * len(shape)
        lo[ax] = slice(0, -1); hi[ax] = slice(1, None)
        lo = tuple(lo); hi = tuple(hi)
        t = _harmonic(kappa[lo], kappa[hi])
        diag[lo] += t; diag[hi] += t
        rows += [idx[lo].ravel(), idx[hi].ravel()]
        cols += [idx[hi].ravel(), idx[lo].ravel()]
        vals += [-t.ravel(), -t.ravel()]
        first = [slice(None)] * len(shape); last = [slice(None)] * len(shape)
        first[ax] = slice(0, 1); last[ax] = slice(-1, None)
        diag[tuple(first)] += 2.0 * kappa[tuple(first)]
        diag[tuple(last)] += 2.0 * kappa[tuple(last)]
    rows.append(idx.ravel()); cols.append(idx.ravel()); vals.append(diag.ravel())
    return _assemble(N, rows, cols, vals)


def lognormal_field(shape, sigma: float, seed: int) -> np.ndarray:
    """kappa = exp(sigma * g), g ~ N(0, 1) i.i.d. per cell from ``default_rng(seed)``."""
    g = np.random.default_rng(seed).standard_normal(int(np.prod(shape)))
    return np.exp(sigma * g).reshape(shape)


def variable_diffusion_2d(n: int, sigma: float = 1.0, seed: int = 3) -> sp.csr_matrix:
    """5-point ``-div(kappa grad u)`` on n x n cells, lognormal kappa, harmonic faces."""
    return _cell_diffusion((n, n), lognormal_field((n, n), sigma, seed))


def variable_diffusion_3d(n: int, sigma: float = 1.0, seed: int = 2) -> sp.csr_matrix:
    """7-point ``-div(kappa grad u)`` on n^3 cells, lognormal kappa, harmonic faces."""
    return _cell_diffusion((n, n, n), lognormal_field((n, n, n), sigma, seed))


def convection_diffusion_2d(n: int, peclet: float = 10.0, angle: float = np.pi / 6) -> sp.csr_matrix:
    """Nonsymmetric ``-lap(u) + w . grad(u)`` on an n x n grid, first-order upwind.

    ``w = peclet * (cos(angle), sin(angle))`` with h = 1 (so ``peclet`` is the cell
    Peclet number); Dirichlet boundary.  Upwinding puts ``|w_d|`` on the diagonal and
    ``-|w_d|`` on the upstream neighbour in each direction d.
    """
    w = (peclet * np.cos(angle), peclet * np.sin(angle))
    I, J = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    I = I.ravel(); J = J.ravel()
    me = I * n + J
    rows, cols, vals = [me], [me], [np.full(n * n, 4.0 + abs(w[0]) + abs(w[1]))]
    for (di, dj) in [(-1, 0), (1, 0), (0, -1), (0, 1)]:
        v = -1.0
        d = 0 if di != 0 else 1
        step = di if di != 0 else dj
        wd = w[d]
        # upstream neighbour: the one the wind comes from (opposite the wind's sign)
        if (wd > 0 and step < 0) or (wd < 0 and step > 0):
            v -= abs(wd)
        ii, jj = I + di, J + dj
        ok = (ii >= 0) & (ii < n) & (jj >= 0) & (jj < n)
        rows.append(me[ok]); cols.append((ii * n + jj)[ok]); vals.append(np.full(ok.sum(), v))
    return _assemble(n * n, rows, cols, vals)
