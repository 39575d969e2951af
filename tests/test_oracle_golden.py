"""The oracle pinned against the reference's own known-answer tests and properties.

Golden values are the literal expectations in AMJax's test-suite:
tests/relaxation/test_relaxation.py:42-101, tests/test_multilevel.py:16-48,50-108,
110-153,155-182,450-478.  The reference itself (JAX + PyAMG) is not importable here.
"""

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import eigsh

from amjax_b200 import amg_setup, gallery
from oracle import amg_oracle as O
from tests.helpers import host_hierarchy, oracle_ml


def _tridiag(n):
    return sp.diags([2 * np.ones(n), -np.ones(n - 1), -np.ones(n - 1)], [0, -1, 1], shape=(n, n), format="csr")


@pytest.mark.parametrize("n,x,b,expect", [
    (1, [0.0], [0.0], [0.0]),
    (3, [0.0, 0.0, 0.0], [0.0, 1.0, 2.0], [0.0, 0.5, 1.0]),
    (3, [0.0, 1.0, 2.0], [0.0, 0.0, 0.0], [0.5, 1.0, 0.5]),
    (1, [0.0], [10.0], [5.0]),
    (3, [0.0, 1.0, 2.0], [10.0, 20.0, 30.0], [5.5, 11.0, 15.5]),
])
def test_jacobi_known_answers(n, x, b, expect):
    A = _tridiag(n)
    out = O.jacobi(A, np.array(x), np.array(b), O.inverse_diagonal(A))
    np.testing.assert_almost_equal(out, expect)


def test_jacobi_omega_third():
    A = _tridiag(3)
    x0 = np.arange(3.0)
    out = O.jacobi(A, x0, np.array([10.0, 20.0, 30.0]), O.inverse_diagonal(A), omega=1.0 / 3.0)
    np.testing.assert_almost_equal(out, 2 / 3 * x0 + 1 / 3 * np.array([5.5, 11.0, 15.5]))


def test_jacobi_dtype_preserved():
    A = gallery.poisson((4,)).astype(np.float32)
    out = O.jacobi(A, np.zeros(4, np.float32), np.arange(4, dtype=np.float32), O.inverse_diagonal(A))
    assert out.dtype == np.float32


def test_spectral_radius_known_answers():
    A = sp.csr_matrix(np.diag(2 * np.ones(4)))
    np.testing.assert_almost_equal(O.approximate_spectral_radius(A, O.inverse_diagonal(A)), 1.0, decimal=5)
    A = gallery.poisson((10,))
    rho = O.approximate_spectral_radius(A, O.inverse_diagonal(A))
    ref = eigsh(sp.diags(1.0 / A.diagonal()) @ A, k=1, which="LM", return_eigenvectors=False)[0]
    assert abs(rho - ref) / ref < 0.1


def test_inverse_diagonal_zero_and_duplicates():
    A = sp.coo_matrix((np.array([1.0, 1.0, 3.0, 5.0]), (np.array([0, 0, 1, 2]), np.array([0, 0, 2, 2]))), shape=(3, 3))
    np.testing.assert_array_equal(O.inverse_diagonal(A), [0.5, 0.0, 0.2])


def test_cycle_complexity_known_answers():
    nnz = [100, 25, 9, 4]
    for L, exp in [(1, (1, 1, 1)), (2, (2.25, 2.25, 2.25)), (3, (2.59, 3.18, 3.18)), (4, (2.72, 3.88, 3.66))]:
        got = tuple(O.cycle_complexity(nnz[:L], c) for c in "VWF")
        np.testing.assert_allclose(got, exp)
    with pytest.raises(NotImplementedError):
        O.cycle_complexity(nnz, "AMLI")


@pytest.mark.parametrize("solver,kw", [("jacobi", {"iterations": 500, "omega": 2 / 3}), ("pinv", {}), ("lu", {}), ("qr", {})])
def test_coarse_solvers(solver, kw):
    for A in [sp.csr_matrix(np.diag(np.arange(1, 5, dtype=float))), gallery.poisson((4,)), gallery.poisson((4, 4))]:
        lvl = O.Level(A)
        cs = O.CoarseSolver(solver, lvl, **kw)
        b = np.arange(A.shape[0], dtype=float)
        x = cs(A, np.zeros_like(b), b)
        np.testing.assert_almost_equal(A @ x, b, decimal=3)


@pytest.mark.parametrize("cycle", ["V", "W", "F"])
@pytest.mark.parametrize("coarse", ["pinv", "lu", "qr", "jacobi"])
def test_solve_converges_rs(cycle, coarse):
    """tests/test_multilevel.py:72-90 (RS, Poisson 20x20, withrho Jacobi, tol 1e-8)."""
    host = host_hierarchy("rs", 20)
    spec = ("jacobi", {"iterations": 1, "withrho": True})
    ml = oracle_ml(host, pre=spec, coarse=coarse)
    b = np.random.default_rng(30459128).random(400)
    x, it = O.solve(ml, b, tol=1e-8, maxiter=100, cycle_type=cycle)
    A = host.levels[0].A
    assert np.linalg.norm(b - A @ x) < 1e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("cycle", ["V", "W", "F"])
def test_pcg_converges(cycle):
    """tests/test_multilevel.py:50-70 (RS 50x50, CG with the AMG preconditioner)."""
    host = host_hierarchy("rs", 50)
    spec = ("jacobi", {"iterations": 1, "withrho": True})
    ml = oracle_ml(host, pre=spec, coarse="jacobi")
    A = host.levels[0].A
    b = np.random.default_rng(1331277597).random(A.shape[0])
    x, _ = O.cg(A, b, tol=1e-8, maxiter=30, M=O.aspreconditioner(ml, cycle))
    assert np.linalg.norm(b - A @ x) < 1e-8 * np.linalg.norm(b)


def test_sa_hierarchy_converges():
    host = host_hierarchy("sa", 50)
    assert len(host.levels) > 1
    ml = oracle_ml(host)
    A = host.levels[0].A
    b = np.random.default_rng(0).standard_normal(A.shape[0])
    x, it = O.solve(ml, b, tol=1e-8, maxiter=100)
    assert np.linalg.norm(b - A @ x) < 1e-8 * np.linalg.norm(b) and it < 60


@pytest.mark.parametrize("cycle", ["V", "W", "F"])
def test_adjoint_matches_central_differences(cycle):
    """tests/test_multilevel.py:155-182: directional derivative of sum(solve(b, A)) w.r.t.
    A equals central finite differences (eps 1e-4, rtol 1e-3)."""
    host = host_hierarchy("rs", 10)
    spec = ("jacobi", {"iterations": 1, "withrho": True})
    ml = oracle_ml(host, pre=spec)
    A = host.levels[0].A.toarray()
    b = np.random.default_rng(42).random(A.shape[0])
    d = np.random.default_rng(0).standard_normal(A.shape)
    f = lambda M: np.sum(O.solve(ml, b, A=sp.csr_matrix(M), tol=1e-10, maxiter=100, cycle_type=cycle)[0])
    x, _ = O.solve(ml, b, A=sp.csr_matrix(A), tol=1e-10, maxiter=100, cycle_type=cycle)
    lam, gA = O.adjoint(ml, x, np.ones_like(b), tol=1e-10, maxiter=100, cycle_type=cycle, A=sp.csr_matrix(A))
    eps = 1e-4
    fd = (f(A + eps * d) - f(A - eps * d)) / (2 * eps)
    np.testing.assert_allclose(np.sum(gA * d), fd, rtol=1e-3)


def test_adjoint_nonsymmetric_needs_transpose():
    """The oracle's adjoint solves A^T lambda = v; on a nonsymmetric operator that (not
    the reference's A lambda = v) matches finite differences."""
    A = gallery.convection_diffusion_2d(12, peclet=2.0)
    host = amg_setup.smoothed_aggregation_solver(A)
    ml = oracle_ml(host)
    b = np.random.default_rng(3).standard_normal(A.shape[0])
    v = np.random.default_rng(4).standard_normal(A.shape[0])
    x, _ = O.solve(ml, b, tol=1e-13, maxiter=400)
    lam, _ = O.adjoint(ml, x, v, tol=1e-13, maxiter=400)
    np.testing.assert_allclose(lam, np.linalg.solve(A.T.toarray(), v), rtol=1e-8, atol=1e-10)
    lam_bad, _ = O.adjoint(ml, x, v, tol=1e-13, maxiter=400, transpose=False)
    assert np.linalg.norm(lam_bad - lam) > 1e-3 * np.linalg.norm(lam)


def test_sampled_grad_equals_dense_on_pattern():
    """tests/test_multilevel.py:209-247: the values-gradient is the dense gradient at the
    pattern."""
    A = gallery.poisson((5, 5))
    rng = np.random.default_rng(0)
    lam, x = rng.standard_normal(25), rng.standard_normal(25)
    g = O.sampled_grad(A, lam, x)
    dense = -np.outer(lam, x)
    coo = A.tocoo()
    np.testing.assert_allclose(g, dense[coo.row, coo.col], rtol=1e-12)


def test_mixed_and_batched_columns_are_independent():
    host = host_hierarchy("sa", 20)
    ml = oracle_ml(host)
    B = np.random.default_rng(9).standard_normal((400, 3))
    for c in range(3):
        x, it = O.solve(ml, B[:, c], tol=1e-8, maxiter=80)
        assert np.linalg.norm(B[:, c] - host.levels[0].A @ x) < 1e-8 * np.linalg.norm(B[:, c])
