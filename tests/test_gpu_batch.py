"""Ragged multi-hierarchy batch (config 3b, scaled down): several SA hierarchies of
different sizes -- isotropic Poisson and rotated anisotropic diffusion -- each with its own
number of right-hand sides, solved by AMG-PCG in ONE graph launch.  Each system's result
must equal its own individual solve (same kernels, deterministic reductions) and reach the
FP64-checked tolerance."""

import numpy as np
import pytest

from amjax_b200 import MultilevelSolver, amg_setup, gallery, pcg_batch

pytestmark = pytest.mark.gpu

W23 = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})


def _systems(count=6, seed=1):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(12, 49))
        k = int(rng.integers(1, 6))
        if i % 2:
            A = gallery.anisotropic_diffusion_2d(n, 1e-2 if (i // 2) % 2 == 0 else 1e-3, np.pi / 4)
        else:
            A = gallery.poisson((n, n))
        B = rng.standard_normal((A.shape[0], k)) if k > 1 else rng.standard_normal(A.shape[0])
        out.append((A, B))
    return out


@pytest.mark.parametrize("precision", ["mixed", "f64"])
def test_batch_equals_individual_solves(precision):
    systems = _systems()
    mls = [MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W23,
                                       postsmoother=W23) for A, _ in systems]
    X, info = pcg_batch(mls, [B for _, B in systems], tol=1e-8, maxiter=400, precision=precision,
                        return_info=True)
    for (A, B), ml, x, inf in zip(systems, mls, X, info):
        xi, ii = ml.pcg(B, tol=1e-8, maxiter=400, precision=precision, return_info=True)
        assert ii["iterations"] == inf["iterations"]
        assert np.linalg.norm(x - xi) <= 1e-14 * np.linalg.norm(xi)
        r = np.linalg.norm((B - A @ x).reshape(A.shape[0], -1), axis=0) / \
            np.linalg.norm(B.reshape(A.shape[0], -1), axis=0)
        assert np.all(r < 1e-8), r


def test_batch_twice_reuses_graph_and_rejects_duplicates():
    systems = _systems(3, seed=2)
    mls = [MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A)) for A, _ in systems]
    rhs = [B for _, B in systems]
    X1 = pcg_batch(mls, rhs, tol=1e-8, maxiter=400)
    X2 = pcg_batch(mls, rhs, tol=1e-8, maxiter=400)
    for a, b in zip(X1, X2):
        assert np.array_equal(a, b)
    with pytest.raises(ValueError):
        pcg_batch([mls[0], mls[0]], [rhs[0], rhs[0]])
