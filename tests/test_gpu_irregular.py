"""GPU parity on irregular operators: weighted graph Laplacians of random geometric graphs
(points uniform in the unit square, edges within a radius, random positive weights, a small
diagonal shift so the matrix is SPD), with irregular row lengths (1-22 nonzeros: isolated
points keep only their diagonal) and smoothed-aggregation hierarchies of four levels with
irregular aggregates, down to a coarsest level of 1-4 rows.

* FP64 standalone solve: iterates after 1, 2 and 5 V-, W- and F-cycles within 1e-10 of the
  oracle's; the same (V, PCG) on a Ruge-Stuben hierarchy of the same operator;
* FP64 PCG: iterates after 1 and 3 steps within 1e-10 of the oracle's CG, and the converged
  iteration count within one of it;
* mixed precision (k = 5): PCG and standalone reach the FP64-checked tolerance 1e-8.
"""

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.spatial import cKDTree

from amjax_b200 import MultilevelSolver, amg_setup
from oracle import amg_oracle as O

from helpers import oracle_ml, rel

pytestmark = pytest.mark.gpu

W = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})


def geometric_laplacian(n, seed, radius_scale=1.0):
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2))
    r = radius_scale * np.sqrt(np.log(n) / (np.pi * n))
    pairs = np.array(sorted(cKDTree(pts).query_pairs(r)), dtype=np.int64).reshape(-1, 2)
    w = rng.uniform(0.5, 2.0, len(pairs))
    Wm = sp.coo_matrix((np.concatenate([w, w]), (np.concatenate([pairs[:, 0], pairs[:, 1]]),
                                                 np.concatenate([pairs[:, 1], pairs[:, 0]]))), shape=(n, n)).tocsr()
    L = sp.diags(np.asarray(Wm.sum(axis=1)).ravel() + 1e-2) - Wm
    L = sp.csr_matrix(L)
    L.sort_indices()
    return L


CASES = [(2000, 1), (6000, 2), (12000, 3)]


@pytest.fixture(scope="module", params=CASES, ids=[f"n{n}-seed{s}" for n, s in CASES])
def problem(request):
    n, seed = request.param
    A = geometric_laplacian(n, seed)
    host = amg_setup.smoothed_aggregation_solver(A)
    ml = MultilevelSolver.from_pyamg(host, presmoother=W, postsmoother=W)
    return A, host, ml, seed


def test_irregular_rows(problem):
    A, host, ml, seed = problem
    deg = np.diff(A.indptr)
    assert deg.max() >= 3 * deg.min()
    assert len(ml.levels) >= 3


@pytest.mark.parametrize("cycle", ["V", "W", "F"])
def test_solve_per_iterate_fp64(problem, cycle):
    A, host, ml, seed = problem
    oml = oracle_ml(host)
    b = np.random.default_rng(seed).standard_normal(A.shape[0])
    hist = []
    O.solve_loop(oml, b, tol=0.0, maxiter=5, cycle_type=cycle, history=hist)
    for m in (1, 2, 5):
        x = ml.solve(b, tol=0.0, maxiter=m, cycle=cycle)
        assert rel(x, hist[m - 1]) < 1e-10, (m, rel(x, hist[m - 1]))


def test_ruge_stuben_per_iterate_fp64(problem):
    A, _, _, seed = problem
    host = amg_setup.ruge_stuben_solver(A)
    ml = MultilevelSolver.from_pyamg(host, presmoother=W, postsmoother=W)
    oml = oracle_ml(host)
    b = np.random.default_rng(seed + 30).standard_normal(A.shape[0])
    hist = []
    O.solve_loop(oml, b, tol=0.0, maxiter=4, cycle_type="V", history=hist)
    for m in (1, 4):
        x = ml.solve(b, tol=0.0, maxiter=m)
        assert rel(x, hist[m - 1]) < 1e-10, (m, rel(x, hist[m - 1]))
    hist = []
    O.cg(A, b, tol=0.0, maxiter=3, M=O.aspreconditioner(oml), history=hist)
    xm = ml.pcg(b, tol=0.0, maxiter=3)
    assert rel(xm, hist[2]) < 1e-10


def test_pcg_per_iterate_fp64(problem):
    A, host, ml, seed = problem
    oml = oracle_ml(host)
    b = np.random.default_rng(seed + 10).standard_normal(A.shape[0])
    hist = []
    xo, ko = O.cg(A, b, tol=1e-8, maxiter=200, M=O.aspreconditioner(oml), history=hist)
    x, info = ml.pcg(b, tol=1e-8, maxiter=200, return_info=True)
    assert abs(info["iterations"][0] - ko) <= 1
    assert rel(x, xo) < 1e-8
    for m in (1, 3):
        xm = ml.pcg(b, tol=0.0, maxiter=m)
        assert rel(xm, hist[m - 1]) < 1e-10, (m, rel(xm, hist[m - 1]))


def test_mixed_reaches_fp64_tolerance(problem):
    A, host, ml, seed = problem
    B = np.random.default_rng(seed + 20).standard_normal((A.shape[0], 5))
    for method in ("pcg", "solve"):
        X, info = getattr(ml, method)(B, tol=1e-8, maxiter=500, precision="mixed", return_info=True)
        r = np.linalg.norm(B - A @ X, axis=0) / np.linalg.norm(B, axis=0)
        assert np.all(r <= 1e-8), (method, r, info["iterations"])
