"""GPU parity: the CUDA solve phase against the FP64 oracle on the same hierarchies.

Bar (FP64): per-iterate relative difference <= 1e-10 and identical iteration counts
(+-1 allowed at the tolerance boundary); FP32 / mixed: FP64-checked residual reaches
the tolerance.  Every call goes through the C ABI (libamg_b200.so).
"""

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from amjax_b200 import MultilevelSolver, jacobi, inverse_diagonal, CSRMatrix
from amjax_b200 import _native as N
from oracle import amg_oracle as O
from tests.helpers import host_hierarchy, oracle_ml, rel

pytestmark = pytest.mark.gpu

W23 = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})


def _ml(kind, n, pre=W23, post=None, coarse="pinv", **kw):
    host = host_hierarchy(kind, n)
    ml = MultilevelSolver.from_pyamg(host, presmoother=pre, postsmoother=pre if post is None else post,
                                     coarse_solver=coarse, **kw)
    return host, ml


# ------------------------------------------------------------------ relaxation KATs
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
    """tests/relaxation/test_relaxation.py:42-73 through the CUDA Jacobi kernel."""
    A = CSRMatrix.from_scipy(_tridiag(n))
    Dinv = inverse_diagonal(A)
    out = jacobi(A, torch.tensor(x, dtype=torch.float64, device="cuda"),
                 torch.tensor(b, dtype=torch.float64, device="cuda"), Dinv)
    np.testing.assert_allclose(out.cpu().numpy(), expect, rtol=0, atol=1e-14)


def test_jacobi_omega_third():
    """tests/relaxation/test_relaxation.py:75-80."""
    A = CSRMatrix.from_scipy(_tridiag(3))
    x0 = torch.arange(3, dtype=torch.float64, device="cuda")
    out = jacobi(A, x0, torch.tensor([10.0, 20.0, 30.0], dtype=torch.float64, device="cuda"),
                 inverse_diagonal(A), omega=1.0 / 3.0)
    np.testing.assert_allclose(out.cpu().numpy(), 2 / 3 * np.arange(3) + 1 / 3 * np.array([5.5, 11.0, 15.5]),
                               atol=1e-14)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("iterations,k", [(1, 1), (3, 1), (2, 5), (1, 8)])
def test_jacobi_vs_oracle(dtype, iterations, k):
    host = host_hierarchy("sa", 40)
    A = host.levels[0].A.astype(dtype)
    rng = np.random.default_rng(7)
    x = rng.standard_normal((A.shape[0], k)).astype(dtype)
    b = rng.standard_normal((A.shape[0], k)).astype(dtype)
    Ad = CSRMatrix.from_scipy(A, dtype=dtype)
    Dinv = inverse_diagonal(Ad)
    xs = x[:, 0] if k == 1 else x
    bs = b[:, 0] if k == 1 else b
    out = jacobi(Ad, torch.as_tensor(xs).cuda(), torch.as_tensor(bs).cuda(), Dinv, iterations=iterations,
                 omega=0.7).cpu().numpy()
    ref = O.jacobi(A, xs.astype(np.float64), bs.astype(np.float64),
                   O.inverse_diagonal(A.astype(np.float64))[:, None] if k > 1 else O.inverse_diagonal(A.astype(np.float64)),
                   iterations, 0.7)
    tol = 1e-13 if dtype == np.float64 else 2e-5
    assert rel(out, ref) < tol


def test_inverse_diagonal_zero_rule():
    """Zero diagonal -> zero (relaxation.py:53-61)."""
    A = sp.csr_matrix(np.array([[2.0, 1.0, 0.0], [0.0, 0.0, 1.0], [0.0, 0.0, 4.0]]))
    d = inverse_diagonal(CSRMatrix.from_scipy(A)).cpu().numpy()
    np.testing.assert_array_equal(d, [0.5, 0.0, 0.25])


# ------------------------------------------------------------------ standalone solve parity
@pytest.mark.parametrize("kind", ["rs", "sa", "rootnode", "pairwise"])
@pytest.mark.parametrize("cycle", ["V", "W", "F"])
def test_solve_per_iterate_fp64(kind, cycle):
    """FP64 iterates equal the oracle's per cycle to <= 1e-10 relative."""
    host, ml = _ml(kind, 40)
    oml = oracle_ml(host)
    b = np.random.default_rng(0).standard_normal(host.levels[0].A.shape[0])
    hist = []
    O.solve_loop(oml, b, tol=0.0, maxiter=6, cycle_type=cycle, history=hist)
    for m in (1, 2, 6):
        x = ml.solve(b, tol=0.0, maxiter=m, cycle=cycle)
        assert rel(x, hist[m - 1]) < 1e-10, (m, rel(x, hist[m - 1]))


def test_config1_rs_poisson100_iterations():
    """2D Poisson 100x100, RS, V, Jacobi 2/3 1+1, pinv, b = ones, tol 1e-10, maxiter 100."""
    host, ml = _ml("rs", 100)
    oml = oracle_ml(host)
    b = np.ones(host.levels[0].A.shape[0])
    xo, ito, rro = O.solve_loop(oml, b, tol=1e-10, maxiter=100)
    x, info = ml.solve(b, tol=1e-10, maxiter=100, return_info=True)
    assert abs(info["iterations"][0] - ito) <= 1
    assert rel(x, xo) < 1e-10
    A = host.levels[0].A
    assert np.linalg.norm(b - A @ x) < 1e-10 * np.linalg.norm(b)


@pytest.mark.parametrize("coarse,kw", [("pinv", {}), ("lu", {}), ("qr", {}), ("jacobi", {"iterations": 20, "omega": 0.8})])
def test_coarse_solvers_parity(coarse, kw):
    host, ml = _ml("rs", 20, coarse=coarse, coarse_solver_kwargs=kw)
    oml = oracle_ml(host, coarse=coarse, coarse_kwargs=kw)
    b = np.random.default_rng(3).random(host.levels[0].A.shape[0])
    hist = []
    O.solve_loop(oml, b, tol=0.0, maxiter=3, history=hist)
    x = ml.solve(b, tol=0.0, maxiter=3)
    assert rel(x, hist[-1]) < 1e-10


def test_batched_freeze_matches_columns():
    """k columns in one launch: each column's iterate and count equal its own solve."""
    host, ml = _ml("sa", 40)
    A = host.levels[0].A
    rng = np.random.default_rng(5)
    B = rng.standard_normal((A.shape[0], 6))
    B[:, 2] *= 1e-6  # converges at a different trip
    B[:, 4] = 0.0    # zero right-hand side: x = 0, no cycle
    X, info = ml.solve(B, tol=1e-8, maxiter=60, return_info=True)
    oml = oracle_ml(host)
    for c in range(B.shape[1]):
        xo, ito, _ = O.solve_loop(oml, B[:, c], tol=1e-8, maxiter=60)
        assert abs(info["iterations"][c] - ito) <= 1
        assert rel(X[:, c], xo) < 1e-10 or np.linalg.norm(xo) == 0.0
    assert info["iterations"][4] == 0 and np.all(X[:, 4] == 0)


@pytest.mark.parametrize("pre,post", [
    (("jacobi", {"iterations": 2, "omega": 0.6}), ("jacobi", {"iterations": 3, "omega": 0.7})),
    (None, ("jacobi", {"iterations": 1, "omega": 2 / 3})),
    (("jacobi", {"iterations": 1, "omega": 2 / 3}), None),
])
def test_smoother_variants(pre, post):
    host, ml = _ml("sa", 30, pre=pre, post=post)
    oml = oracle_ml(host, pre=pre, post=post)
    b = np.random.default_rng(1).standard_normal(host.levels[0].A.shape[0])
    for cycle in "VW":
        hist = []
        O.solve_loop(oml, b, tol=0.0, maxiter=3, cycle_type=cycle, history=hist)
        x = ml.solve(b, tol=0.0, maxiter=3, cycle=cycle)
        assert rel(x, hist[-1]) < 1e-10


# ------------------------------------------------------------------ preconditioner / PCG
@pytest.mark.parametrize("cycle", ["V", "W", "F"])
def test_preconditioner_parity(cycle):
    host, ml = _ml("sa", 40)
    oml = oracle_ml(host)
    b = np.random.default_rng(2).standard_normal(host.levels[0].A.shape[0])
    M = ml.aspreconditioner(cycle=cycle)
    z = M(b)
    assert rel(z, O.aspreconditioner(oml, cycle)(b)) < 1e-12


@pytest.mark.parametrize("kind", ["sa", "rs"])
def test_pcg_parity_fp64(kind):
    host, ml = _ml(kind, 50)
    oml = oracle_ml(host)
    A = host.levels[0].A
    b = np.random.default_rng(1331).random(A.shape[0])
    hist = []
    xo, ko = O.cg(A, b, tol=1e-8, maxiter=30, M=O.aspreconditioner(oml), history=hist)
    x, info = ml.pcg(b, tol=1e-8, maxiter=30, return_info=True)
    assert abs(info["iterations"][0] - ko) <= 1
    assert rel(x, xo) < 1e-9
    assert np.linalg.norm(b - A @ x) < 1e-8 * np.linalg.norm(b)
    for m in (1, 3):
        xm = ml.pcg(b, tol=0.0, maxiter=m)
        assert rel(xm, hist[m - 1]) < 1e-10


@pytest.mark.parametrize("k", [1, 4, 16])
def test_mixed_precision_reaches_fp64_tolerance(k):
    host, ml = _ml("sa", 60)
    A = host.levels[0].A
    B = np.random.default_rng(0).standard_normal((A.shape[0], k))
    b = B[:, 0] if k == 1 else B
    for method in ("solve", "pcg"):
        x = getattr(ml, method)(b, tol=1e-10, maxiter=200, precision="mixed")
        r = np.linalg.norm((b - A @ x).reshape(A.shape[0], -1), axis=0) / np.linalg.norm(b.reshape(A.shape[0], -1), axis=0)
        assert np.all(r < 1e-10), (method, r)


def test_fp32_hierarchy_runs_in_fp32():
    """dtype=float32 keeps FP32 end to end (tests/test_multilevel.py:402-435) and its
    iterates follow the FP64 oracle to FP32 accuracy."""
    host = host_hierarchy("sa", 30)
    ml = MultilevelSolver.from_pyamg(host, dtype=np.float32)
    b = torch.ones(host.levels[0].A.shape[0], dtype=torch.float32, device="cuda")
    x = ml.solve(b, tol=1e-4, maxiter=20)
    assert x.dtype == torch.float32
    oml = oracle_ml(host, pre=("jacobi", {"iterations": 1, "omega": 1.0}))
    xo, _, _ = O.solve_loop(oml, np.ones(host.levels[0].A.shape[0]), tol=1e-4, maxiter=20)
    assert rel(x.cpu().numpy(), xo) < 1e-4
    M = ml.aspreconditioner()
    assert M(b).dtype == torch.float32


def test_launch_counter_counts():
    host, ml = _ml("sa", 20)
    before = N.kernel_launch_count()
    ml.solve(np.ones(host.levels[0].A.shape[0]), tol=1e-8, maxiter=20)
    assert N.kernel_launch_count() > before


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_spectral_radius_on_device_matches_host(dtype):
    """The GPU power iteration (same start vector, same 15 steps) agrees with the host
    estimate the reference's set-up uses (relaxation.py:101-132) to rounding."""
    from amjax_b200.relaxation.relaxation import approximate_spectral_radius
    from amjax_b200 import gallery
    A = CSRMatrix.from_scipy(gallery.poisson((60, 70)), dtype=dtype)
    Dinv = inverse_diagonal(A)
    host = approximate_spectral_radius(A, Dinv)
    dev = approximate_spectral_radius(A, Dinv, on_device=True)
    tol = 1e-12 if dtype == np.float64 else 1e-5
    assert abs(dev - host) <= tol * host
    assert abs(O.approximate_spectral_radius(A.to_scipy(), O.inverse_diagonal(A.to_scipy())) - dev) <= tol * host
