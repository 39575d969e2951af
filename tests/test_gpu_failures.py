"""Failure detection without a GPU fault: every failure here is made on the host.

* Bad CSR structure handed straight to the C ABI (no Python-side validation in between):
  row pointers that decrease, do not start at 0 or do not end at nnz, and column indices
  out of range are refused with AMG_ERR_BAD_MATRIX by amg_hierarchy_create, by the A0
  override of amg_pcg / amg_solve, and by the stand-alone kernels.  Columns that are not
  sorted within a row are valid (the kernels do not need them sorted) and give the same
  product as sorted ones.
* A NaN in one right-hand-side column stops that column at once (NaN compares false in
  the stop rules, as in the reference's while-loop, amjax/multilevel.py:414-422, and in
  jax.scipy.sparse.linalg.cg); the other columns converge exactly as without it.
* maxiter exhaustion is silent, as in the reference (multilevel.py:414-425): iterations ==
  maxiter and relres > tol come back in ``return_info``, with no exception.
* A right-hand side of the wrong length is a ValueError; an ``out`` of the wrong size is
  refused.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from amjax_b200 import MultilevelSolver, amg_setup, gallery
from amjax_b200 import _native as N
from tests.helpers import rel

pytestmark = pytest.mark.gpu

W23 = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})


def _raw_csr(indptr, indices, data, shape, nnz=None):
    """An amg_csr descriptor over device copies of the given arrays, taken as they are."""
    keep = [torch.as_tensor(np.asarray(indptr, dtype=np.int32)).cuda(),
            torch.as_tensor(np.asarray(indices, dtype=np.int32)).cuda(),
            torch.as_tensor(np.asarray(data, dtype=np.float64)).cuda()]
    d = N.amg_csr()
    d.n_rows, d.n_cols = shape
    d.nnz = len(indices) if nnz is None else nnz
    d.rowptr = keep[0].data_ptr()
    d.col = keep[1].data_ptr()
    d.val64 = keep[2].data_ptr()
    d.val32 = None
    return d, keep


def _poisson_parts(n=10):
    A = gallery.poisson((n, n)).tocsr()
    return A.indptr.copy(), A.indices.copy(), A.data.copy(), A.shape


def _corruptions():
    ip, ix, dv, shape = _poisson_parts()
    out = {}
    bad = ip.copy(); bad[4], bad[5] = bad[5], bad[4]
    out["decreasing rowptr"] = (bad, ix, dv, shape, None)
    bad = ip.copy(); bad[0] = 1
    out["rowptr[0] != 0"] = (bad, ix, dv, shape, None)
    out["rowptr[n] != nnz"] = (ip, ix[:-3], dv[:-3], shape, None)
    bad = ix.copy(); bad[17] = shape[1]
    out["column too large"] = (ip, bad, dv, shape, None)
    bad = ix.copy(); bad[3] = -1
    out["negative column"] = (ip, bad, dv, shape, None)
    return out


@pytest.mark.parametrize("case", list(_corruptions()))
def test_standalone_kernels_refuse_bad_structure(case):
    ip, ix, dv, shape, nnz = _corruptions()[case]
    d, keep = _raw_csr(ip, ix, dv, shape, nnz)
    lib = N.load()
    x = torch.ones(shape[1], dtype=torch.float64, device="cuda")
    y = torch.zeros(shape[0], dtype=torch.float64, device="cuda")
    st = lib.amg_spmv(C.byref(d), 0, N.ptr(x), N.ptr(y), 1, N.stream_ptr())
    assert st == 5, (case, st, lib.amg_last_error())
    assert torch.all(y == 0)  # nothing ran
    st = lib.amg_inverse_diagonal(C.byref(d), 0, N.ptr(y), N.stream_ptr())
    assert st == 5


def test_hierarchy_create_refuses_bad_operator():
    A = gallery.poisson((24, 24))
    host = amg_setup.smoothed_aggregation_solver(A)
    ml = MultilevelSolver.from_pyamg(host, presmoother=W23, postsmoother=W23)
    descs, coarse = ml._native_descs()
    lib = N.load()
    h = C.c_void_p()
    assert lib.amg_hierarchy_create(descs, len(descs), C.byref(coarse), C.byref(h)) == 0
    lib.amg_hierarchy_destroy(h)
    # level 1's prolongation with one column index past the coarse size
    P = ml.levels[1].P if len(ml.levels) > 2 else ml.levels[0].P
    lvl = 1 if len(ml.levels) > 2 else 0
    col = P.col.clone()
    col[5] = P.shape[1] + 3
    descs[lvl].P.col = col.data_ptr()
    h2 = C.c_void_p()
    st = lib.amg_hierarchy_create(descs, len(descs), C.byref(coarse), C.byref(h2))
    assert st == 5, lib.amg_last_error()
    assert b"P" in lib.amg_last_error() and b"column" in lib.amg_last_error()


def test_a0_override_refuses_bad_structure():
    A = gallery.poisson((20, 20))
    ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W23, postsmoother=W23)
    H = A.tocsr()
    bad = H.indices.copy()
    bad[40] = A.shape[1]
    d, keep = _raw_csr(H.indptr, bad, H.data, A.shape)
    b = torch.ones(A.shape[0], dtype=torch.float64, device="cuda")
    x = torch.zeros_like(b)
    lib = N.load()
    it = (C.c_int32 * 1)()
    rr = (C.c_double * 1)()
    st = lib.amg_pcg(ml._native(), N.PREC_F64, N.ptr(b), N.ptr(x), 1, 1e-8, 0.0, 50, 0, 1, C.byref(d), it, rr,
                     N.stream_ptr())
    assert st == 5, lib.amg_last_error()
    st = lib.amg_solve(ml._native(), N.PREC_F64, N.ptr(b), N.ptr(x), 1, 1e-8, 50, 0, 1, C.byref(d), it, rr,
                       N.stream_ptr())
    assert st == 5
    # the handle is still usable afterwards
    xg = ml.pcg(b, tol=1e-8, maxiter=50)
    assert np.linalg.norm(A @ xg.cpu().numpy() - 1.0) < 1e-7 * np.sqrt(A.shape[0])


def test_unsorted_columns_are_valid():
    H = gallery.poisson((16, 16)).tocsr()
    ip, ix, dv = H.indptr, H.indices.copy(), H.data.copy()
    for i in range(H.shape[0]):  # reverse every row's column order
        s, e = ip[i], ip[i + 1]
        ix[s:e] = ix[s:e][::-1].copy()
        dv[s:e] = dv[s:e][::-1].copy()
    d, keep = _raw_csr(ip, ix, dv, H.shape)
    xh = np.random.default_rng(0).standard_normal((H.shape[1], 4))
    x = torch.as_tensor(xh).cuda()
    y = torch.zeros(H.shape[0], 4, dtype=torch.float64, device="cuda")
    N.call("amg_spmv", C.byref(d), 0, N.ptr(x), N.ptr(y), 4, N.stream_ptr())
    np.testing.assert_allclose(y.cpu().numpy(), H @ xh, rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("precision", ["f64", "mixed", "mixed-f64cg"])
@pytest.mark.parametrize("method", ["solve", "pcg"])
def test_nan_column_stops_alone(method, precision):
    A = gallery.poisson((40, 40))
    ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W23, postsmoother=W23)
    B = np.random.default_rng(3).standard_normal((A.shape[0], 4))
    Bn = B.copy()
    Bn[7, 2] = np.nan
    f = getattr(ml, method)
    x, info = f(Bn, tol=1e-9, maxiter=200, precision=precision, return_info=True)
    assert info["iterations"][2] == 0
    assert np.all(x[:, 2] == 0.0)
    good = [0, 1, 3]
    xr, ir = f(B[:, good], tol=1e-9, maxiter=200, precision=precision, return_info=True)
    # k = 4 and k = 3 launch different layouts, so the column sums may round differently
    for c, ic in zip(good, ir["iterations"]):
        assert abs(info["iterations"][c] - ic) <= 1
    assert rel(x[:, good], xr) < (1e-12 if precision == "f64" else 1e-6)
    r = np.linalg.norm(B[:, good] - A @ x[:, good], axis=0) / np.linalg.norm(B[:, good], axis=0)
    assert np.all(r <= 1e-9)


@pytest.mark.parametrize("precision", ["f64", "mixed", "mixed-f64cg", "f32"])
@pytest.mark.parametrize("method", ["solve", "pcg"])
def test_maxiter_exhaustion_is_silent(method, precision):
    A = gallery.poisson((48, 48))
    dtype = np.float32 if precision == "f32" else np.float64
    ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W23, postsmoother=W23,
                                     dtype=dtype)
    B = np.random.default_rng(4).standard_normal((A.shape[0], 3)).astype(dtype)
    x, info = getattr(ml, method)(B, tol=1e-13, maxiter=2, precision=precision, return_info=True)
    assert list(info["iterations"]) == [2, 2, 2]
    r = np.linalg.norm(B - A @ x.astype(np.float64), axis=0) / np.linalg.norm(B, axis=0)
    assert np.all(r > 1e-13) and np.all(np.asarray(info["relres"]) > 1e-13)


def test_wrong_sizes_are_refused():
    A = gallery.poisson((20, 20))
    ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W23, postsmoother=W23)
    with pytest.raises(ValueError):
        ml.solve(np.ones(A.shape[0] + 1))
    with pytest.raises(ValueError):
        ml.pcg(np.ones((A.shape[0] - 1, 2)))
    with pytest.raises(ValueError):
        ml.pcg(torch.ones(A.shape[0] + 2, dtype=torch.float64, device="cuda"))
    out = torch.empty(A.shape[0], 3, dtype=torch.float64)
    with pytest.raises(RuntimeError):
        ml.pcg(np.ones((A.shape[0], 2)), out=out)
