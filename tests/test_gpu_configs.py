"""GPU parity at the workload sizes of the benchmark, through the C ABI.

* Poisson 500 x 500 (N = 250,000), smoothed aggregation, V-cycle, Jacobi omega = 2/3 1+1,
  pinv: the headline hierarchy.  FP64 standalone solve and FP64 PCG, one right-hand side
  (``default_rng(0).standard_normal(N)``) and 64 (``default_rng(0).standard_normal((N, 64))``,
  stored [N, 64]).  Iterates after 1 and 3 cycles / CG steps and the converged solution
  agree with the FP64 oracle to <= 1e-10 relative; iteration counts agree within +-1 (the
  oracle runs column by column on a few of the 64 columns).  The mixed-precision forms
  reach the FP64-checked tolerance 1e-8.
* Variable-coefficient diffusion 256 x 256 (lognormal kappa, sigma 1, seed 3), k = 16:
  dL/db and dL/dvalues of L = 1/2 ||x - x*||^2 through SA V-cycle PCG (FP64, tol 1e-10)
  against central differences (h = 1e-6) in random directions, <= 1e-6 relative.
* Upwind convection-diffusion 256 x 256 (Peclet 10, 30 degree wind) on an AIR hierarchy:
  the same gradient checks with the adjoint solve on the explicit transposed hierarchy.
* 3D lognormal diffusion 48^3: FP64 and mixed solves to 1e-10 against a direct FP64
  solve, and FP64 V/W/F iterates against the oracle.
* ``x0`` warm starts of ``solve`` and ``pcg`` (amjax/multilevel.py:384-394) and their
  gradients with respect to A.

Reference loop and stopping rule: amjax/multilevel.py:407-425; adjoint: :428-444;
finite-difference protocol: tests/test_multilevel.py:155-182.
"""

import functools

import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

from amjax_b200 import CSRMatrix, MultilevelSolver, SparseA, amg_setup, gallery
from oracle import amg_oracle as O
from tests.helpers import rel

pytestmark = pytest.mark.gpu

W23 = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})
COLS = (0, 21, 42, 63)   # columns of the k = 64 block the oracle checks


def _dev(a):
    return torch.as_tensor(np.asarray(a), dtype=torch.float64, device="cuda")


@functools.lru_cache(maxsize=None)
def _poisson500():
    A = gallery.poisson((500, 500))
    host = amg_setup.smoothed_aggregation_solver(A)
    ml = MultilevelSolver.from_pyamg(host, presmoother=W23, postsmoother=W23, coarse_solver="pinv")
    oml = O.Hierarchy.from_host(host, presmoother=W23, postsmoother=W23, coarse_solver="pinv")
    return A, ml, oml


@functools.lru_cache(maxsize=None)
def _rhs(k):
    n = 250_000
    rng = np.random.default_rng(0)
    return rng.standard_normal(n) if k == 1 else rng.standard_normal((n, k))


def _oracle_cols(k):
    B = _rhs(k)
    return [(0, B)] if k == 1 else [(c, B[:, c]) for c in COLS]


# ------------------------------------------------------------------ headline hierarchy, FP64
@pytest.mark.parametrize("k", [1, 64])
def test_poisson500_standalone_fp64_matches_oracle(k):
    A, ml, oml = _poisson500()
    B = _rhs(k)
    X, info = ml.solve(B, tol=1e-8, maxiter=100, return_info=True)
    X1 = ml.solve(B, tol=0.0, maxiter=1)
    X3 = ml.solve(B, tol=0.0, maxiter=3)
    X = X.reshape(A.shape[0], -1)
    X1 = X1.reshape(A.shape[0], -1)
    X3 = X3.reshape(A.shape[0], -1)
    for c, b in _oracle_cols(k):
        hist = []
        xo, ito, rro = O.solve_loop(oml, b, tol=1e-8, maxiter=100, history=hist)
        assert abs(info["iterations"][c] - ito) <= 1, (c, info["iterations"][c], ito)
        assert rel(X[:, c], xo) <= 1e-10, (c, rel(X[:, c], xo))
        assert rel(X1[:, c], hist[0]) <= 1e-10
        assert rel(X3[:, c], hist[2]) <= 1e-10
    r = np.linalg.norm(B.reshape(A.shape[0], -1) - A @ X, axis=0) / np.linalg.norm(B.reshape(A.shape[0], -1), axis=0)
    assert np.all(r < 1e-8), r.max()


@pytest.mark.parametrize("k", [1, 64])
def test_poisson500_pcg_fp64_matches_oracle(k):
    A, ml, oml = _poisson500()
    B = _rhs(k)
    X, info = ml.pcg(B, tol=1e-8, maxiter=100, return_info=True)
    X1 = ml.pcg(B, tol=0.0, maxiter=1).reshape(A.shape[0], -1)
    X3 = ml.pcg(B, tol=0.0, maxiter=3).reshape(A.shape[0], -1)
    X = X.reshape(A.shape[0], -1)
    M = O.aspreconditioner(oml)
    for c, b in _oracle_cols(k):
        hist = []
        xo, ko = O.cg(A, b, tol=1e-8, maxiter=100, M=M, history=hist)
        assert abs(info["iterations"][c] - ko) <= 1, (c, info["iterations"][c], ko)
        assert rel(X[:, c], xo) <= 1e-10, (c, rel(X[:, c], xo))
        assert rel(X1[:, c], hist[0]) <= 1e-10
        assert rel(X3[:, c], hist[2]) <= 1e-10
    r = np.linalg.norm(B.reshape(A.shape[0], -1) - A @ X, axis=0) / np.linalg.norm(B.reshape(A.shape[0], -1), axis=0)
    assert np.all(r < 1e-8), r.max()


@pytest.mark.parametrize("method", ["solve", "pcg"])
@pytest.mark.parametrize("k", [1, 64])
def test_poisson500_mixed_reaches_fp64_tolerance(method, k):
    """FP32 cycle with FP64 outer work: the FP64-checked residual reaches 1e-8 in every
    column, and the solution is as close to the FP64 path's as the tolerance allows."""
    A, ml, _ = _poisson500()
    B = _rhs(k)
    X = getattr(ml, method)(B, tol=1e-8, maxiter=100, precision="mixed").reshape(A.shape[0], -1)
    X64 = getattr(ml, method)(B, tol=1e-8, maxiter=100).reshape(A.shape[0], -1)
    Bm = B.reshape(A.shape[0], -1)
    r = np.linalg.norm(Bm - A @ X, axis=0) / np.linalg.norm(Bm, axis=0)
    assert np.all(r < 1e-8), r.max()
    assert rel(X, X64) < 1e-6


# ------------------------------------------------------------------ gradients at 256 x 256
def _fd_check(loss, B0, vals0, rng, h=1e-6, rtol=1e-6):
    """Gradients of loss(B, values) against central differences in one random direction
    for B and one for the values (scaled by |values|, so every entry moves relatively)."""
    Bt = _dev(B0).requires_grad_(True)
    vt = _dev(vals0).requires_grad_(True)
    gb, gv = torch.autograd.grad(loss(Bt, vt, 1e-10), (Bt, vt))
    db = rng.standard_normal(B0.shape)
    dv = rng.standard_normal(vals0.shape) * np.abs(vals0)
    with torch.no_grad():
        f = lambda Bm, vv: float(loss(_dev(Bm), _dev(vv), 1e-14))
        fd_b = (f(B0 + h * db, vals0) - f(B0 - h * db, vals0)) / (2 * h)
        fd_v = (f(B0, vals0 + h * dv) - f(B0, vals0 - h * dv)) / (2 * h)
    np.testing.assert_allclose(float(torch.sum(gb * _dev(db))), fd_b, rtol=rtol)
    np.testing.assert_allclose(float(gv.cpu().numpy() @ dv), fd_v, rtol=rtol)
    return gb, gv


def test_diffusion256_k16_gradients_match_central_differences():
    """L = 1/2 ||x - x*||^2, x solving A(kappa) X = B for 16 right-hand sides on 2D lognormal
    diffusion 256 x 256 (kappa from seed 3; B and x* ~ N(0,1)), SA V-cycle PCG in FP64 to
    1e-10.  The finite differences use solves to 1e-14 so their own error stays far below h."""
    n, k = 256, 16
    A = gallery.variable_diffusion_2d(n, sigma=1.0, seed=3)
    host = amg_setup.smoothed_aggregation_solver(A)
    ml = MultilevelSolver.from_pyamg(host, presmoother=W23, postsmoother=W23)
    rng = np.random.default_rng(3)
    B0 = rng.standard_normal((A.shape[0], k))
    Xs = _dev(rng.standard_normal((A.shape[0], k)))
    pattern = CSRMatrix.from_scipy(A)

    def loss(Bm, vv, tol):
        x = ml.pcg(Bm, A=SparseA(pattern, vv), tol=tol, maxiter=500)
        return 0.5 * torch.sum((x - Xs) ** 2)

    gb, _ = _fd_check(loss, B0, A.data.copy(), rng)
    # dL/db is the adjoint solution A^-T (x - x*): check one column against a direct solve
    x = ml.pcg(_dev(B0), tol=1e-12, maxiter=500)
    lam = spla.splu(A.T.tocsc()).solve((x - Xs)[:, 3].cpu().numpy())
    assert rel(gb[:, 3].cpu().numpy(), lam) < 1e-6


def test_air_convection_diffusion256_gradients():
    """Upwind convection-diffusion 256 x 256 (Peclet 10, 30 degree wind), AIR hierarchy
    (R != P^T), k = 4, standalone AIR V-cycle in FP64: the backward solve runs on the
    explicit transposed hierarchy; gradients against central differences <= 1e-6."""
    n, k = 256, 4
    C = gallery.convection_diffusion_2d(n, peclet=10.0, angle=np.pi / 6)
    host = amg_setup.air_solver(C)
    ml = MultilevelSolver.from_pyamg(host, presmoother=W23, postsmoother=W23)
    assert ml.transposed() is not ml
    rng = np.random.default_rng(3)
    B0 = rng.standard_normal((C.shape[0], k))
    Xs = _dev(rng.standard_normal((C.shape[0], k)))
    pattern = CSRMatrix.from_scipy(C)

    def loss(Bm, vv, tol):
        x = ml.solve(Bm, A=SparseA(pattern, vv), tol=tol, maxiter=600)
        return 0.5 * torch.sum((x - Xs) ** 2)

    gb, _ = _fd_check(loss, B0, C.data.copy(), rng)
    x = ml.solve(_dev(B0), tol=1e-13, maxiter=600)
    lam = spla.splu(C.T.tocsc()).solve((x - Xs)[:, 1].cpu().numpy())
    assert rel(gb[:, 1].cpu().numpy(), lam) < 1e-6


# ------------------------------------------------------------------ 3D, 48^3
@functools.lru_cache(maxsize=None)
def _cube48():
    A = gallery.variable_diffusion_3d(48, sigma=1.0, seed=2)
    host = amg_setup.smoothed_aggregation_solver(A)
    ml = MultilevelSolver.from_pyamg(host, presmoother=W23, postsmoother=W23)
    return A, host, ml


def test_cube48_error_against_direct_solve():
    """3D lognormal diffusion 48^3 (N = 110,592): FP64 and FP32-cycle refinement solves to
    1e-10 both land within 1e-8 of a direct FP64 solve, and within 1e-9 of each other."""
    A, _, ml = _cube48()
    b = np.random.default_rng(2).standard_normal(A.shape[0])
    xd = spla.splu(A.tocsc()).solve(b)
    x64 = ml.solve(b, tol=1e-10, maxiter=300)
    xmx = ml.solve(b, tol=1e-10, maxiter=300, precision="mixed")
    assert rel(x64, xd) < 1e-8 and rel(xmx, xd) < 1e-8, (rel(x64, xd), rel(xmx, xd))
    assert rel(xmx, x64) < 1e-9


@pytest.mark.parametrize("cycle", ["V", "W", "F"])
def test_cube48_cycles_match_oracle(cycle):
    A, host, ml = _cube48()
    oml = O.Hierarchy.from_host(host, presmoother=W23, postsmoother=W23)
    b = np.random.default_rng(2).standard_normal(A.shape[0])
    hist = []
    O.solve_loop(oml, b, tol=0.0, maxiter=4, cycle_type=cycle, history=hist)
    for m in (1, 4):
        assert rel(ml.solve(b, tol=0.0, maxiter=m, cycle=cycle), hist[m - 1]) <= 1e-10


# ------------------------------------------------------------------ x0 warm starts
def test_x0_warm_start_solve_and_pcg():
    """solve(b, x0=...) shifts b by A x0 and adds x0 back (multilevel.py:384-394): the
    result equals the oracle's per iterate; pcg with x0 converges from the shifted start."""
    A = gallery.poisson((60, 60))
    host = amg_setup.smoothed_aggregation_solver(A)
    ml = MultilevelSolver.from_pyamg(host, presmoother=W23, postsmoother=W23)
    oml = O.Hierarchy.from_host(host, presmoother=W23, postsmoother=W23)
    rng = np.random.default_rng(4)
    b = rng.standard_normal(A.shape[0])
    x0 = rng.standard_normal(A.shape[0])
    for m in (1, 3):
        xo, _ = O.solve(oml, b, x0=x0, tol=0.0, maxiter=m)
        assert rel(ml.solve(b, x0=x0, tol=0.0, maxiter=m), xo) <= 1e-10
    x, info = ml.solve(b, x0=x0, tol=1e-9, maxiter=100, return_info=True)
    xo, ito = O.solve(oml, b, x0=x0, tol=1e-9, maxiter=100)
    assert abs(info["iterations"][0] - ito) <= 1 and rel(x, xo) <= 1e-10
    # pcg: the oracle's cg from the same start
    M = O.aspreconditioner(oml)
    for m in (1, 3):
        xo, _ = O.cg(A, b - A @ x0, tol=0.0, maxiter=m, M=M)
        assert rel(ml.pcg(b, x0=x0, tol=0.0, maxiter=m), xo + x0) <= 1e-10
    x = ml.pcg(b, x0=x0, tol=1e-10, maxiter=100)
    assert np.linalg.norm(b - A @ x) <= 1.01e-10 * np.linalg.norm(b - A @ x0)


@pytest.mark.parametrize("sparse", [False, True])
def test_x0_gradient_with_respect_to_A(sparse):
    """With x0 the gradient with respect to A is -lambda x^T for the FULL solution x (the
    term through b - A x0 included): checked against central differences."""
    host = amg_setup.smoothed_aggregation_solver(gallery.poisson((12, 12)))
    ml = MultilevelSolver.from_pyamg(host, presmoother=W23, postsmoother=W23)
    H = host.levels[0].A
    rng = np.random.default_rng(9)
    b = _dev(rng.standard_normal(H.shape[0]))
    x0 = _dev(rng.standard_normal(H.shape[0]) * 3.0)
    w = _dev(rng.standard_normal(H.shape[0]))
    pattern = CSRMatrix.from_scipy(H)

    def f(a, tol):
        A = SparseA(pattern, a) if sparse else a
        return torch.sum(w * ml.solve(b, A=A, x0=x0, tol=tol, maxiter=300))

    a0 = H.data.copy() if sparse else H.toarray()
    at = _dev(a0).requires_grad_(True)
    (g,) = torch.autograd.grad(f(at, 1e-13), at)
    d = rng.standard_normal(a0.shape) * (np.abs(a0) if sparse else 1.0)
    h = 1e-6
    with torch.no_grad():
        fd = (float(f(_dev(a0 + h * d), 1e-14)) - float(f(_dev(a0 - h * d), 1e-14))) / (2 * h)
    np.testing.assert_allclose(float(torch.sum(g * _dev(d))), fd, rtol=1e-6)
