"""Property-based GPU tests of the fused CSR kernels on random sparsity patterns.

Random square CSR matrices (hypothesis, derandomised): 1-600 rows, empty rows, short rows
and a few long rows (up to a full row), random values; k right-hand sides from 1 to 72
(odd counts, counts that are not a multiple of the vector width, more than 64); FP64 and
FP32; the autotuned layout or one forced kernel family (AMG_KB_G, as in
test_gpu_kernel_variants.py).  Checked through the C ABI:

* `amg_spmv` (y = A x) against a float64 product of the same (dtype-rounded) values, within
  the forward error bound of a sum of len(row) products, (len + 1) u (|A| |x|)_i;
* one `amg_jacobi` sweep against a float64 sweep (relaxation.py:94-96), within
  (len + 4) u (omega |d| (|b| + |A| |x|) + 2 |x|)_i.

Rows with no nonzeros give exactly zero (SpMV) and the D^-1 = 0 rule's x (Jacobi).
"""

import os

import numpy as np
import pytest
import scipy.sparse as sp
import torch
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

from amjax_b200 import CSRMatrix, inverse_diagonal
from amjax_b200 import _native as N

pytestmark = pytest.mark.gpu

FAMILIES = [None, "8", "16", "65", "66", "80", "129", "130", "136", "196", "200", "260", "264"]


@st.composite
def cases(draw):
    n = draw(st.integers(1, 600))
    k = draw(st.sampled_from([1, 2, 3, 5, 8, 13, 16, 24, 64, 72]))
    seed = draw(st.integers(0, 2**31 - 1))
    dt = draw(st.sampled_from([np.float64, np.float32]))
    family = draw(st.sampled_from(FAMILIES))
    rng = np.random.default_rng(seed)
    kind = rng.choice(3, size=n, p=[0.15, 0.8, 0.05])
    lens = np.where(kind == 0, 0, np.where(kind == 1, rng.integers(1, 9, n), rng.integers(9, max(n, 9) + 1, n)))
    lens = np.minimum(lens, n)
    indptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    cols = [np.sort(rng.choice(n, int(m), replace=False)) for m in lens]
    indices = np.concatenate(cols) if indptr[-1] else np.zeros(0, dtype=np.int64)
    data = rng.standard_normal(int(indptr[-1]))
    A = sp.csr_matrix((data, indices, indptr), shape=(n, n))
    return A, k, dt, family, seed


def _call_with_family(family, fn):
    old = os.environ.get("AMG_KB_G")
    try:
        if family is None:
            os.environ.pop("AMG_KB_G", None)
        else:
            os.environ["AMG_KB_G"] = family
        return fn()
    finally:
        if old is None:
            os.environ.pop("AMG_KB_G", None)
        else:
            os.environ["AMG_KB_G"] = old


SETTINGS = settings(max_examples=60, deadline=None, derandomize=True,
                    suppress_health_check=[HealthCheck.too_slow, HealthCheck.data_too_large])


@SETTINGS
@given(cases())
def test_spmv_random_patterns(case):
    A, k, dt, family, seed = case
    n = A.shape[0]
    M = CSRMatrix.from_scipy(A)
    tdt = torch.float64 if dt == np.float64 else torch.float32
    g = torch.Generator(device="cuda").manual_seed(seed % (2**31))
    x = torch.randn(n, k, dtype=tdt, device="cuda", generator=g)
    y = torch.full((n, k), float("nan"), dtype=tdt, device="cuda")

    def run():
        N.call("amg_spmv", M.desc(), 0 if dt == np.float64 else 1, N.ptr(x), N.ptr(y), k, N.stream_ptr())
        torch.cuda.synchronize()

    _call_with_family(family, run)
    vals = A.data.astype(dt).astype(np.float64)
    Ar = sp.csr_matrix((vals, A.indices, A.indptr), shape=A.shape)
    xh = x.double().cpu().numpy()
    ref = Ar @ xh
    bound = (np.diff(A.indptr)[:, None] + 1) * np.finfo(dt).eps * (abs(Ar) @ np.abs(xh)) + 1e-300
    got = y.double().cpu().numpy()
    assert np.isfinite(got).all()
    err = np.abs(got - ref)
    assert (err <= bound).all(), (family, k, dt, float((err / bound).max()))
    empty = np.diff(A.indptr) == 0
    assert (got[empty] == 0).all()


@SETTINGS
@given(cases())
def test_jacobi_random_patterns(case):
    A, k, dt, family, seed = case
    n = A.shape[0]
    A = A + sp.diags(np.where(np.arange(n) % 7 == 3, 0.0, 4.0 + np.abs(A).sum(axis=1).A1))  # some zero diagonals
    A = sp.csr_matrix(A)
    A.sort_indices()
    M = CSRMatrix.from_scipy(A)
    tdt = torch.float64 if dt == np.float64 else torch.float32
    dinv = inverse_diagonal(M).to(tdt)
    g = torch.Generator(device="cuda").manual_seed(seed % (2**31) + 1)
    x = torch.randn(n, k, dtype=tdt, device="cuda", generator=g)
    b = torch.randn(n, k, dtype=tdt, device="cuda", generator=g)
    y = torch.full((n, k), float("nan"), dtype=tdt, device="cuda")
    omega = 2.0 / 3.0

    def run():
        N.call("amg_jacobi", M.desc(), 0 if dt == np.float64 else 1, N.ptr(x), N.ptr(b), N.ptr(dinv), N.ptr(y),
               k, 1, float(omega), N.stream_ptr())
        torch.cuda.synchronize()

    _call_with_family(family, run)
    vals = A.data.astype(dt).astype(np.float64)
    Ar = sp.csr_matrix((vals, A.indices, A.indptr), shape=A.shape)
    xh, bh = x.double().cpu().numpy(), b.double().cpu().numpy()
    d = dinv.double().cpu().numpy()[:, None]
    om = float(np.asarray(omega, dtype=dt))
    ref = (1 - om) * xh + om * (d * (bh - Ar @ xh) + xh)
    lens = np.diff(A.indptr)[:, None]
    bound = (lens + 4) * np.finfo(dt).eps * (om * np.abs(d) * (np.abs(bh) + abs(Ar) @ np.abs(xh)) + 2 * np.abs(xh)) + 1e-300
    got = y.double().cpu().numpy()
    assert np.isfinite(got).all()
    err = np.abs(got - ref)
    assert (err <= bound).all(), (family, k, dt, float((err / bound).max()))
