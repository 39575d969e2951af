"""GPU tests of the mixed-precision PCG in its reliable-update form (precision='mixed').

The CG vectors are FP32; the FP64 solution and the FP64 true residual b - A x are
refreshed whenever the FP32 residual has dropped by a fixed factor and before any column
stops, so every column's stop rule (jax.scipy.sparse.linalg.cg's <r, r> <=
max(tol^2 <b, b>, atol^2), as the reference's benchmark calls it,
benchmarks/benchmark.ipynb cell 7) is decided on the FP64 residual.  Checked against the
plain FP64 PCG and the FP64-CG-around-FP32-cycle form ('mixed-f64cg') on the same
hierarchy: FP64-checked residuals reach the tolerance, iteration counts stay within two
of FP64's, solutions agree to the tolerance's accuracy, maxiter exhaustion reports the
true residual, and zero / NaN columns retire at once without touching the others.  (With
one right-hand side 'mixed' runs the FP64-CG form, the faster one there.)
"""

import numpy as np
import pytest

from amjax_b200 import MultilevelSolver, amg_setup, gallery
from tests.helpers import rel

pytestmark = pytest.mark.gpu

W23 = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})


def _ml(n=60, kind="poisson"):
    A = gallery.poisson((n, n)) if kind == "poisson" else gallery.variable_diffusion_2d(n, sigma=1.0, seed=3)
    ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W23, postsmoother=W23)
    return A, ml


def _relres(A, B, X):
    n = A.shape[0]
    B = np.asarray(B).reshape(n, -1)
    X = np.asarray(X).reshape(n, -1)
    return np.linalg.norm(B - A @ X, axis=0) / np.linalg.norm(B, axis=0)


@pytest.mark.parametrize("kind", ["poisson", "lognormal"])
@pytest.mark.parametrize("k", [1, 4, 16])
@pytest.mark.parametrize("tol", [1e-8, 1e-10])
def test_reliable_pcg_reaches_fp64_tolerance(kind, k, tol):
    A, ml = _ml(64, kind)
    B = np.random.default_rng(5).standard_normal((A.shape[0], k))
    b = B[:, 0] if k == 1 else B
    x64, i64 = ml.pcg(b, tol=tol, maxiter=300, return_info=True)
    xru, iru = ml.pcg(b, tol=tol, maxiter=300, precision="mixed", return_info=True)
    xfc, ifc = ml.pcg(b, tol=tol, maxiter=300, precision="mixed-f64cg", return_info=True)
    for x in (xru, xfc):
        assert np.all(_relres(A, b, x) <= tol), _relres(A, b, x).max()
    for c in range(k):
        assert abs(iru["iterations"][c] - i64["iterations"][c]) <= 2, (iru["iterations"], i64["iterations"])
        assert iru["relres"][c] <= tol
    # the reported relres of the reliable form is the FP64 true residual of the returned x
    # (at 1e-10 the two summation orders of b - A x differ by ~1e-6 relative); with k = 1
    # 'mixed' runs the FP64-CG form, which reports its recursive residual
    if k > 1:
        np.testing.assert_allclose(iru["relres"], _relres(A, b, xru), rtol=1e-4)
    assert rel(xru, x64) < 1e3 * tol


def test_reliable_pcg_maxiter_reports_true_residual():
    """maxiter exhaustion is silent (the reference returns x, amjax/multilevel.py:414-425):
    every column stops at maxiter with its FP64 true residual reported."""
    A, ml = _ml(64)
    B = np.random.default_rng(6).standard_normal((A.shape[0], 8))
    x, info = ml.pcg(B, tol=1e-14, maxiter=3, precision="mixed", return_info=True)
    assert info["iterations"] == [3] * 8
    r = _relres(A, B, x)
    assert np.all(r > 1e-14)
    np.testing.assert_allclose(info["relres"], r, rtol=1e-4)
    # the same three CG steps as the FP64 path, to FP32 accuracy
    x64 = ml.pcg(B, tol=1e-14, maxiter=3)
    assert rel(x, x64) < 1e-5


def test_reliable_pcg_zero_and_nan_columns_retire_alone():
    A, ml = _ml(48)
    B = np.random.default_rng(7).standard_normal((A.shape[0], 6))
    B[:, 1] = 0.0
    B[5, 4] = np.nan
    x, info = ml.pcg(B, tol=1e-9, maxiter=200, precision="mixed", return_info=True)
    assert info["iterations"][1] == 0 and np.all(x[:, 1] == 0.0)
    assert info["iterations"][4] == 0
    good = [0, 2, 3, 5]
    assert np.all(_relres(A, B[:, good], x[:, good]) <= 1e-9)
    ref = ml.pcg(B[:, good], tol=1e-9, maxiter=200, precision="mixed")
    assert rel(x[:, good], ref) < 1e-6


def test_reliable_pcg_batch_matches_single_solves():
    import torch
    from amjax_b200 import pcg_batch
    systems = [_ml(n)[1] for n in (40, 56, 72)]
    rhs = [torch.as_tensor(np.random.default_rng(20 + i).standard_normal((m.levels[0].A.shape[0], k))).cuda()
           for i, (m, k) in enumerate(zip(systems, (1, 3, 8)))]
    X, info = pcg_batch(systems, rhs, tol=1e-9, maxiter=200, precision="mixed", return_info=True)
    for m, b, x, inf in zip(systems, rhs, X, info):
        xs, i1 = m.pcg(b, tol=1e-9, maxiter=200, precision="mixed", return_info=True)
        assert torch.equal(x.reshape(xs.shape), xs)
        assert list(inf["iterations"]) == list(i1["iterations"])


@pytest.mark.parametrize("kind", ["poisson", "lognormal"])
@pytest.mark.parametrize("k", [1, 8])
def test_reliable_standalone_solve(kind, k):
    """The mixed standalone solve in its reliable-update form: FP32 residual and increment
    updated after every cycle, FP64 refreshes, columns stopping on the FP64 norm with the
    reference's rule (amjax/multilevel.py:414-422): iterations within one of the FP64
    solve's, the tolerance reached on the FP64 residual, the reported relres the true one;
    maxiter exhaustion stops every column at maxiter with its true residual."""
    A, ml = _ml(64, kind)
    B = np.random.default_rng(9).standard_normal((A.shape[0], k))
    b = B[:, 0] if k == 1 else B
    x64, i64 = ml.solve(b, tol=1e-9, maxiter=300, return_info=True)
    x, inf = ml.solve(b, tol=1e-9, maxiter=300, precision="mixed", return_info=True)
    r = _relres(A, b, x)
    assert np.all(r < 1e-9), r.max()
    for c in range(k):
        assert abs(inf["iterations"][c] - i64["iterations"][c]) <= 1, (inf["iterations"], i64["iterations"])
    np.testing.assert_allclose(inf["relres"], r, rtol=1e-4)
    assert rel(x, x64) < 1e-6
    xm, im = ml.solve(b, tol=1e-14, maxiter=4, precision="mixed", return_info=True)
    assert im["iterations"] == [4] * k
    np.testing.assert_allclose(im["relres"], _relres(A, b, xm), rtol=1e-4)
    assert rel(xm, ml.solve(b, tol=1e-14, maxiter=4)) < 1e-5
