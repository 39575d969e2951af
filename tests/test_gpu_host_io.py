"""PCG with host right-hand sides and solution (amg_pcg_host, reached by
MultilevelSolver.pcg for a host [N, k >= 2] block): the k columns are solved in column
blocks whose copies overlap the other block's solve.  Columns are independent, so each
block's result is exactly the device solve of those columns (same plan, same kernels):
checked bit for bit, with odd k (uneven blocks), pinned and unpinned inputs, numpy in /
numpy out, a pinned `out`, and the reported iterations and residuals."""

import numpy as np
import pytest
import torch

from amjax_b200 import MultilevelSolver, amg_setup, gallery

pytestmark = pytest.mark.gpu

W23 = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})


@pytest.mark.parametrize("precision", ["f64", "mixed", "mixed-f64cg"])
@pytest.mark.parametrize("k", [16, 19])
def test_host_block_pcg_equals_device_blocks(precision, k):
    A = gallery.poisson((48, 48))
    ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W23, postsmoother=W23)
    B = np.random.default_rng(k).standard_normal((A.shape[0], k))
    X, info = ml.pcg(B, tol=1e-9, maxiter=200, precision=precision, return_info=True)
    assert isinstance(X, np.ndarray) and X.shape == B.shape
    kc = (k + 1) // 2
    for c0 in (0, kc):
        Bd = torch.as_tensor(np.ascontiguousarray(B[:, c0:c0 + kc])).cuda()
        Xd, inf = ml.pcg(Bd, tol=1e-9, maxiter=200, precision=precision, return_info=True)
        assert np.array_equal(X[:, c0:c0 + kc], Xd.cpu().numpy())
        assert info["iterations"][c0:c0 + kc] == list(inf["iterations"])
    r = np.linalg.norm(B - A @ X, axis=0) / np.linalg.norm(B, axis=0)
    assert np.all(r <= 1e-9)


def test_host_block_pcg_pinned_out_and_torch_input():
    A = gallery.poisson((40, 40))
    ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W23, postsmoother=W23)
    B = torch.as_tensor(np.random.default_rng(2).standard_normal((A.shape[0], 32))).pin_memory()
    out = torch.empty_like(B).pin_memory()
    r = ml.pcg(B, tol=1e-8, maxiter=200, precision="mixed", out=out)
    assert r is out
    X2 = ml.pcg(B.clone(), tol=1e-8, maxiter=200, precision="mixed")  # unpinned CPU tensor in, CPU tensor out
    assert isinstance(X2, torch.Tensor) and not X2.is_cuda
    assert torch.equal(out, X2)
    Xd = ml.pcg(B.cuda(), tol=1e-8, maxiter=200, precision="mixed")
    rel = float(torch.linalg.norm(out - Xd.cpu()) / torch.linalg.norm(Xd.cpu()))
    assert rel < 1e-6  # one k = 32 solve vs two k = 16 blocks: same columns, rounding of the sums


@pytest.mark.parametrize("method", ["pcg", "solve"])
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_odd_k_runs_padded_to_the_vector_width(method, precision):
    """k above 8 and not a multiple of 8 runs on ceil(k / 8) * 8 columns, the extra ones
    zero (they retire at once): the k returned columns equal those of an explicit
    zero-padded solve bit for bit, with the same iterations."""
    A = gallery.poisson((40, 40))
    ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W23, postsmoother=W23)
    B = np.random.default_rng(4).standard_normal((A.shape[0], 21))
    Bp = np.zeros((A.shape[0], 24))
    Bp[:, :21] = B
    f = getattr(ml, method)
    x, inf = f(torch.as_tensor(B).cuda(), tol=1e-9, maxiter=200, precision=precision, return_info=True)
    xp, infp = f(torch.as_tensor(Bp).cuda(), tol=1e-9, maxiter=200, precision=precision, return_info=True)
    assert x.shape == (A.shape[0], 21)
    assert torch.equal(x, xp[:, :21])
    assert list(inf["iterations"]) == list(infp["iterations"])[:21]
    assert list(infp["iterations"])[21:] == [0, 0, 0]


def test_host_block_pcg_refuses_f32_and_null():
    import ctypes as C
    from amjax_b200 import _native as N
    A = gallery.poisson((20, 20))
    ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W23, postsmoother=W23)
    B = torch.zeros(A.shape[0], 4, dtype=torch.float64).pin_memory()
    X = torch.empty_like(B).pin_memory()
    lib = N.load()
    st = lib.amg_pcg_host(ml._native(), N.PREC_F32, N.ptr(B), N.ptr(X), 4, 2, 1e-8, 0.0, 10, 0, 1, None, None,
                          N.stream_ptr())
    assert st == 2
    st = lib.amg_pcg_host(ml._native(), N.PREC_F64, None, N.ptr(X), 4, 2, 1e-8, 0.0, 10, 0, 1, None, None,
                          N.stream_ptr())
    assert st == 1
    st = lib.amg_pcg_host(ml._native(), N.PREC_F64, N.ptr(B), N.ptr(X), 4, 0, 1e-8, 0.0, 10, 0, 1, None, None,
                          N.stream_ptr())
    assert st == 1
