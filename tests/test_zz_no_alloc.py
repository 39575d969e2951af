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
    tol = 1e-13 if dtype == np.float64 else 2e-5
    for call, iterations in enumerate((3, 2)):  # two calls in a row share the scratch array
        x = torch.randn(shape, dtype=tdt, device="cuda", generator=gen)
        b = torch.randn(shape, dtype=tdt, device="cuda", generator=gen)
        ref = _call("amg_jacobi", A, x, b, dinv, k, iterations, 0.7)
        got = _call("amg_jacobi_noalloc", A, x, b, dinv, k, iterations, 0.7)
        err = (torch.linalg.norm((got - ref).double()) / torch.linalg.norm(ref.double())).item()
        assert err <= tol, (call, err)


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
