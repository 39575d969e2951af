"""GPU tests of the hand-written adjoint (amjax/multilevel.py:428-444 and the gradient
tests at tests/test_multilevel.py:155-320), through torch.autograd and the C ABI.

The backward solve runs A^T lambda = v on the transposed hierarchy (the reference solves
A lambda = v, correct only for symmetric A); gradients with respect to A's stored values
come from the library's sampled-outer-product kernel.
"""

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from amjax_b200 import CSRMatrix, MultilevelSolver, SparseA, amg_setup, gallery
from tests.helpers import host_hierarchy

pytestmark = pytest.mark.gpu

RHO = ("jacobi", {"iterations": 1, "withrho": True})
W23 = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})


def _dev(a):
    return torch.as_tensor(np.asarray(a), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("cycle", ["V", "W", "F"])
def test_vjp_dense_A_matches_central_differences(cycle):
    """tests/test_multilevel.py:155-182: directional derivative of sum(solve(b, A)) in a
    random direction equals central differences (eps 1e-4, rtol 1e-3)."""
    host = host_hierarchy("rs", 10)
    ml = MultilevelSolver.from_pyamg(host, presmoother=RHO, postsmoother=RHO)
    A0 = host.levels[0].A.toarray()
    b = _dev(np.random.default_rng(42).random(A0.shape[0]))
    d = np.random.default_rng(0).standard_normal(A0.shape)
    A = _dev(A0).requires_grad_(True)
    f = torch.sum(ml.solve(b, A=A, tol=1e-10, maxiter=100, cycle=cycle))
    (g,) = torch.autograd.grad(f, A)
    assert g.shape == A.shape

    def fval(M):
        with torch.no_grad():
            return float(torch.sum(ml.solve(b, A=_dev(M), tol=1e-10, maxiter=100, cycle=cycle)))

    eps = 1e-4
    fd = (fval(A0 + eps * d) - fval(A0 - eps * d)) / (2 * eps)
    np.testing.assert_allclose(float(torch.sum(g * _dev(d))), fd, rtol=1e-3)


def test_values_gradient_equals_dense_gradient_at_pattern():
    """tests/test_multilevel.py:209-247: the gradient w.r.t. the stored values equals the
    dense gradient read at the pattern (rtol 1e-10)."""
    host = host_hierarchy("rs", 5)
    ml = MultilevelSolver.from_pyamg(host, presmoother=RHO, postsmoother=RHO)
    H = host.levels[0].A
    b = _dev(np.random.default_rng(42).random(H.shape[0]))
    pattern = CSRMatrix.from_scipy(H)
    vals = _dev(H.data).requires_grad_(True)
    (gv,) = torch.autograd.grad(torch.sum(ml.solve(b, A=SparseA(pattern, vals), tol=1e-10, maxiter=100)), vals)
    A = _dev(H.toarray()).requires_grad_(True)
    (gd,) = torch.autograd.grad(torch.sum(ml.solve(b, A=A, tol=1e-10, maxiter=100)), A)
    coo = H.tocoo()
    np.testing.assert_allclose(gv.cpu().numpy(), gd.cpu().numpy()[coo.row, coo.col], rtol=1e-10, atol=1e-10)


def test_pcg_values_gradient_equals_dense_gradient():
    """tests/test_multilevel.py:249-290 with the fused PCG in place of jax cg."""
    host = host_hierarchy("rs", 5)
    ml = MultilevelSolver.from_pyamg(host, presmoother=RHO, postsmoother=RHO)
    H = host.levels[0].A
    b = _dev(np.random.default_rng(42).random(H.shape[0]))
    vals = _dev(H.data).requires_grad_(True)
    (gv,) = torch.autograd.grad(torch.sum(ml.pcg(b, A=SparseA(CSRMatrix.from_scipy(H), vals), tol=1e-12,
                                                 maxiter=30)), vals)
    A = _dev(H.toarray()).requires_grad_(True)
    (gd,) = torch.autograd.grad(torch.sum(ml.pcg(b, A=A, tol=1e-12, maxiter=30)), A)
    coo = H.tocoo()
    np.testing.assert_allclose(gv.cpu().numpy(), gd.cpu().numpy()[coo.row, coo.col], rtol=1e-9, atol=1e-11)


def test_gradient_descent_decreases_loss():
    """tests/test_multilevel.py:292-320, and the whole descent trajectory equals the
    oracle's (same losses step by step).  The step is 1e-6: the dense rank-one update
    -lr * lambda x^T leaves A's pattern, and at 1e-4 it makes the fixed hierarchy's
    Jacobi-smoothed cycle diverge on this problem (the oracle diverges identically)."""
    from oracle import amg_oracle as O
    host = host_hierarchy("rs", 10)
    ml = MultilevelSolver.from_pyamg(host, presmoother=RHO, postsmoother=RHO)
    oml = O.Hierarchy.from_host(host, presmoother=RHO, postsmoother=RHO)
    H = host.levels[0].A
    bn = np.random.default_rng(42).random(H.shape[0])
    b = _dev(bn)
    target = torch.ones_like(b)
    A = _dev(H.toarray())
    An = H.toarray()
    lr = 1e-6

    def loss(M):
        return torch.sum((ml.solve(b, A=M, tol=1e-10, maxiter=100) - target) ** 2)

    losses, oracle_losses = [float(loss(A))], []
    for _ in range(5):
        A = A.detach().requires_grad_(True)
        (g,) = torch.autograd.grad(loss(A), A)
        assert torch.isfinite(g).all()
        A = A - lr * g
        losses.append(float(loss(A.detach())))
    for _ in range(6):
        xo, _ = O.solve(oml, bn, A=sp.csr_matrix(An), tol=1e-10, maxiter=100)
        oracle_losses.append(float(np.sum((xo - 1) ** 2)))
        _, gA = O.adjoint(oml, xo, 2 * (xo - 1), tol=1e-10, maxiter=100, A=sp.csr_matrix(An))
        An = An - lr * gA
    assert all(np.isfinite(losses)) and all(b_ < a_ for a_, b_ in zip(losses, losses[1:])), losses
    np.testing.assert_allclose(losses, oracle_losses, rtol=1e-8)


def test_grad_b_is_adjoint_solution():
    host = host_hierarchy("sa", 20)
    ml = MultilevelSolver.from_pyamg(host, presmoother=W23, postsmoother=W23)
    H = host.levels[0].A
    rng = np.random.default_rng(5)
    b = _dev(rng.standard_normal(H.shape[0])).requires_grad_(True)
    v = rng.standard_normal(H.shape[0])
    x = ml.solve(b, tol=1e-12, maxiter=200)
    (gb,) = torch.autograd.grad(torch.sum(x * _dev(v)), b)
    lam = np.linalg.solve(H.T.toarray(), v)
    np.testing.assert_allclose(gb.cpu().numpy(), lam, rtol=1e-8, atol=1e-10)


def test_nonsymmetric_adjoint_uses_transposed_hierarchy():
    """Upwind convection-diffusion (Peclet 10, 30 degree wind): lambda solves A^T lambda = v
    (the reference's A lambda = v would be wrong here); values gradient vs central
    differences (h = 1e-6) to 1e-6 relative."""
    n = 16
    C = gallery.convection_diffusion_2d(n, peclet=10.0, angle=np.pi / 6)
    host = amg_setup.smoothed_aggregation_solver(C)
    ml = MultilevelSolver.from_pyamg(host, presmoother=W23, postsmoother=W23)
    assert ml.transposed() is not ml
    rng = np.random.default_rng(7)
    b = _dev(rng.standard_normal(C.shape[0]))
    v = rng.standard_normal(C.shape[0])
    pattern = CSRMatrix.from_scipy(C)
    vals0 = C.data.copy()
    vals = _dev(vals0).requires_grad_(True)
    x = ml.solve(b, A=SparseA(pattern, vals), tol=1e-14, maxiter=2000)
    (gv,) = torch.autograd.grad(torch.sum(x * _dev(v)), vals)
    xs = np.linalg.solve(C.toarray(), b.cpu().numpy())
    lam = np.linalg.solve(C.T.toarray(), v)
    coo = C.tocoo()
    np.testing.assert_allclose(gv.cpu().numpy(), -lam[coo.row] * xs[coo.col], rtol=1e-6, atol=1e-9)
    h = 1e-6
    dirn = rng.standard_normal(vals0.shape)

    def f(vv):
        with torch.no_grad():
            xx = ml.solve(b, A=SparseA(pattern, _dev(vv)), tol=1e-14, maxiter=2000)
            return float(torch.sum(xx * _dev(v)))

    fd = (f(vals0 + h * dirn) - f(vals0 - h * dirn)) / (2 * h)
    np.testing.assert_allclose(float(gv.cpu().numpy() @ dirn), fd, rtol=1e-6)


def test_batched_diffusion_gradients_match_central_differences():
    """Config-5 style (scaled to 48 x 48): L = 1/2 ||x - x*||^2, x solving A(kappa) x = b for
    k = 4 right-hand sides, lognormal kappa, SA V-cycle PCG in FP64; dL/db and dL/dvalues
    against central differences (h = 1e-6) in random directions, to 1e-6 relative."""
    n, k = 48, 4
    A = gallery.variable_diffusion_2d(n, sigma=1.0, seed=3)
    host = amg_setup.smoothed_aggregation_solver(A)
    ml = MultilevelSolver.from_pyamg(host, presmoother=W23, postsmoother=W23)
    rng = np.random.default_rng(3)
    B0 = rng.standard_normal((A.shape[0], k))
    Xs = _dev(rng.standard_normal((A.shape[0], k)))
    pattern = CSRMatrix.from_scipy(A)
    vals0 = A.data.copy()

    def L(Bm, vv, grad=False):
        x = ml.pcg(Bm, A=SparseA(pattern, vv), tol=1e-14, maxiter=400)
        return 0.5 * torch.sum((x - Xs) ** 2)

    Bt = _dev(B0).requires_grad_(True)
    vt = _dev(vals0).requires_grad_(True)
    gb, gv = torch.autograd.grad(L(Bt, vt), (Bt, vt))
    h = 1e-6
    db = rng.standard_normal(B0.shape)
    dv = rng.standard_normal(vals0.shape) * np.abs(vals0)
    with torch.no_grad():
        fd_b = (float(L(_dev(B0 + h * db), _dev(vals0))) - float(L(_dev(B0 - h * db), _dev(vals0)))) / (2 * h)
        fd_v = (float(L(_dev(B0), _dev(vals0 + h * dv))) - float(L(_dev(B0), _dev(vals0 - h * dv)))) / (2 * h)
    np.testing.assert_allclose(float(torch.sum(gb * _dev(db))), fd_b, rtol=1e-6)
    np.testing.assert_allclose(float(gv.cpu().numpy() @ dv), fd_v, rtol=1e-6)


def test_air_convection_diffusion_gradients():
    """Config 5b (scaled to 64 x 64): upwind convection-diffusion, Peclet 10, 30 degree
    wind, AIR hierarchy (R != P^T), k = 4 right-hand sides, L = 1/2 ||x - x*||^2 with x from
    the standalone AIR V-cycle solve in FP64.  The backward solve runs on the explicit
    transposed hierarchy (A^T, P' = R^T, R' = P^T); dL/db and dL/dvalues match central
    differences (h = 1e-6) to 1e-6 relative, and dL/db equals A^-T (x - x*)."""
    n, k = 64, 4
    C = gallery.convection_diffusion_2d(n, peclet=10.0, angle=np.pi / 6)
    host = amg_setup.air_solver(C)
    ml = MultilevelSolver.from_pyamg(host, presmoother=W23, postsmoother=W23)
    assert ml.transposed() is not ml
    rng = np.random.default_rng(3)
    B0 = rng.standard_normal((C.shape[0], k))
    Xs = _dev(rng.standard_normal((C.shape[0], k)))
    pattern = CSRMatrix.from_scipy(C)
    vals0 = C.data.copy()

    def L(Bm, vv):
        x = ml.solve(Bm, A=SparseA(pattern, vv), tol=1e-13, maxiter=400)
        return 0.5 * torch.sum((x - Xs) ** 2), x

    Bt = _dev(B0).requires_grad_(True)
    vt = _dev(vals0).requires_grad_(True)
    loss, x = L(Bt, vt)
    gb, gv = torch.autograd.grad(loss, (Bt, vt))
    lam = np.linalg.solve(C.T.toarray(), (x - Xs).detach().cpu().numpy())
    np.testing.assert_allclose(gb.cpu().numpy(), lam, rtol=1e-7, atol=1e-10)
    h = 1e-6
    db = rng.standard_normal(B0.shape)
    dv = rng.standard_normal(vals0.shape) * np.abs(vals0)
    with torch.no_grad():
        f = lambda Bm, vv: float(L(_dev(Bm), _dev(vv))[0])
        fd_b = (f(B0 + h * db, vals0) - f(B0 - h * db, vals0)) / (2 * h)
        fd_v = (f(B0, vals0 + h * dv) - f(B0, vals0 - h * dv)) / (2 * h)
    np.testing.assert_allclose(float(torch.sum(gb * _dev(db))), fd_b, rtol=1e-6)
    np.testing.assert_allclose(float(gv.cpu().numpy() @ dv), fd_v, rtol=1e-6)


@pytest.mark.parametrize("factory", ["smoothed_aggregation_solver", "rootnode_solver", "pairwise_solver",
                                     "ruge_stuben_solver", "air_solver"])
def test_from_pyamg_compatibility(factory):
    """tests/test_multilevel.py:322-333: all five factories the reference lists."""
    A = gallery.poisson((20, 20))
    assert len(MultilevelSolver.from_pyamg(getattr(amg_setup, factory)(A), coarse_solver="jacobi").levels) > 1
    ml = MultilevelSolver.from_pyamg(getattr(amg_setup, factory)(A), presmoother=RHO, postsmoother=RHO,
                                     coarse_solver="jacobi")
    b = np.ones(A.shape[0])
    x = ml.solve(b, tol=1e-8, maxiter=300)
    assert np.linalg.norm(b - A @ x) < 1e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("method", ["solve", "pcg"])
def test_adjoint_entry_point_equals_two_calls(method):
    """amg_adjoint (the backward solve plus the sampled dL/dA in one call) gives exactly the
    transposed-hierarchy solve followed by amg_sampled_outer, and rejects F32 and a
    gradient request without a pattern."""
    import ctypes as C
    from amjax_b200 import _native as N
    from amjax_b200.autograd import adjoint, sampled_outer
    A = gallery.convection_diffusion_2d(24, peclet=10.0, angle=np.pi / 6) if method == "solve" else \
        gallery.variable_diffusion_2d(24, sigma=1.0, seed=3)
    host = amg_setup.air_solver(A) if method == "solve" else amg_setup.smoothed_aggregation_solver(A)
    ml = MultilevelSolver.from_pyamg(host, presmoother=RHO, postsmoother=RHO)
    mlt = ml.transposed()
    pattern = CSRMatrix.from_scipy(A)
    rng = np.random.default_rng(8)
    gx = torch.as_tensor(rng.standard_normal((A.shape[0], 3))).cuda()
    x = torch.as_tensor(rng.standard_normal((A.shape[0], 3))).cuda()
    opts = dict(tol=1e-10, atol=0.0, maxiter=400, cycle="V", cycles_per_level=1, precision=None, method=method)
    lam, grad = adjoint(mlt, opts, gx, x, None, pattern)
    f = mlt.pcg if method == "pcg" else mlt.solve
    lam2 = f(gx, tol=1e-10, maxiter=400)
    assert torch.equal(lam, lam2)
    assert torch.equal(grad, sampled_outer(pattern, lam2, x))
    lib = N.load()
    iters = (C.c_int32 * 3)()
    rel = (C.c_double * 3)()
    out = torch.empty_like(gx)
    g = torch.empty(pattern.nnz, dtype=torch.float64, device="cuda")
    st = lib.amg_adjoint(mlt._native(), N.PREC_F32, 0, N.ptr(gx), N.ptr(x), 3, 1e-8, 0.0, 10, 0, 1, None,
                         C.byref(pattern.desc()), N.ptr(out), N.ptr(g), iters, rel, N.stream_ptr())
    assert st == 2
    st = lib.amg_adjoint(mlt._native(), N.PREC_F64, 0, N.ptr(gx), N.ptr(x), 3, 1e-8, 0.0, 10, 0, 1, None, None,
                         N.ptr(out), N.ptr(g), iters, rel, N.stream_ptr())
    assert st == 1
