"""amg_jacobi_noalloc: the allocation-free Jacobi entry point, called through the C ABI.

Callers such as a JAX/XLA custom call (XLA has reserved the GPU's memory up front) or an
application on a fixed memory budget cannot allocate device memory when they call the
library; this entry point keeps the iterate between sweeps in a fixed 16 MiB array
compiled into the library.  Its output must equal the allocating ``amg_jacobi``'s on two
calls in a row (the second call sees the first call's leftovers in the shared array).
Collected last so that a run stopping at the first failure has run everything else.
"""

import numpy as np
import pytest
import torch

from amjax_b200 import CSRMatrix, gallery, inverse_diagonal
from amjax_b200 import _native as N

pytestmark = pytest.mark.gpu


def _call(name, A, x, b, dinv, k, iterations, omega):
    out = torch.empty_like(x)
    dt = 0 if x.dtype == torch.float64 else 1
    N.call(name, A.desc(), dt, N.ptr(x), N.ptr(b), N.ptr(dinv), N.ptr(out), k, iterations, omega, N.stream_ptr())
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("dtype,k", [(np.float64, 1), (np.float32, 1), (np.float64, 8), (np.float32, 16)])
def test_noalloc_matches_allocating_entry_point(dtype, k):
    A = CSRMatrix.from_scipy(gallery.poisson((40, 40)), dtype=dtype)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    dinv = inverse_diagonal(A).to(tdt)
    gen = torch.Generator(device="cuda").manual_seed(11)
    shape = (A.shape[0],) if k == 1 else (A.shape[0], k)
    for call, iterations in enumerate((3, 2)):  # two calls in a row share the scratch array
        x = torch.randn(shape, dtype=tdt, device="cuda", generator=gen)
        b = torch.randn(shape, dtype=tdt, device="cuda", generator=gen)
        ref = _call("amg_jacobi", A, x, b, dinv, k, iterations, 0.7)
        got = _call("amg_jacobi_noalloc", A, x, b, dinv, k, iterations, 0.7)
        # the same kernels in the same order: the outputs are bit-identical
        assert torch.equal(got, ref), (call, (got - ref).abs().max().item())


@pytest.mark.parametrize("name", ["amg_jacobi", "amg_jacobi_noalloc"])
def test_jacobi_rejects_aliasing_and_bad_dtype(name):
    """out aliasing x, b or dinv would let a later sweep read what an earlier one wrote;
    an unknown dtype is refused before anything is copied, also with iterations = 0."""
    A = CSRMatrix.from_scipy(gallery.poisson((8, 8)))
    dinv = inverse_diagonal(A)
    x = torch.zeros(A.shape[0], dtype=torch.float64, device="cuda")
    b = torch.ones_like(x)
    for out in (x, b, dinv):
        st = getattr(N.load(), name)(A.desc(), 0, N.ptr(x), N.ptr(b), N.ptr(dinv), N.ptr(out), 1, 2, 0.7,
                                     N.stream_ptr())
        assert st == 1
    out = torch.full_like(x, 5.0)
    for iterations in (0, 2):
        st = getattr(N.load(), name)(A.desc(), 2, N.ptr(x), N.ptr(b), N.ptr(dinv), N.ptr(out), 1, iterations,
                                     0.7, N.stream_ptr())
        assert st == 1 and "dtype" in N.load().amg_last_error().decode()
    torch.cuda.synchronize()
    assert torch.all(out == 5.0)


def test_noalloc_rejects_oversize():
    A = CSRMatrix.from_scipy(gallery.poisson((1100, 1100)))  # 1.21M rows: 2 FP64 columns > 16 MiB
    dinv = inverse_diagonal(A)
    x = torch.zeros(A.shape[0], 2, dtype=torch.float64, device="cuda")
    with pytest.raises(N.NativeError) as ei:
        _call("amg_jacobi_noalloc", A, x, x.clone(), dinv, 2, 2, 0.7)
    assert ei.value.status == 1 and "16777216" in str(ei.value)
    # one sweep needs no scratch, so the same size is accepted
    out = _call("amg_jacobi_noalloc", A, x, x.clone(), dinv, 2, 1, 0.7)
    assert torch.all(out == 0)
