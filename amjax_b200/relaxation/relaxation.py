"""Relaxation primitives (amjax/relaxation/relaxation.py) on the B200 kernels.

``jacobi`` runs the fused CSR Jacobi kernel; ``inverse_diagonal`` and
``approximate_spectral_radius`` are set-up helpers.  The spectral-radius estimate runs
on the host in numpy by default, exactly as the reference's (15 power steps from
``default_rng(0)``), so a resolved ``omega`` is the same number the reference bakes in;
``on_device=True`` runs the same steps on the GPU.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

from .. import _native as N
from ..csr import CSRMatrix


def _host_csr(A):
    if isinstance(A, CSRMatrix):
        return A.to_scipy()
    if sp.issparse(A):
        return sp.csr_matrix(A)
    if isinstance(A, torch.Tensor):
        return sp.csr_matrix(A.detach().cpu().numpy())
    return sp.csr_matrix(np.asarray(A))


def matrix_diagonal(A):
    """Diagonal of A as a 1-D array: the sum of stored (i, i) entries
    (relaxation.py:9-33; duplicates add, as the reference's scatter-add does)."""
    H = sp.coo_matrix(_host_csr(A))
    m = H.row == H.col
    d = np.zeros(H.shape[0], dtype=H.dtype)
    np.add.at(d, H.row[m], H.data[m])
    return d


def inverse_diagonal(A):
    """Element-wise inverse of the diagonal, zero where the diagonal is zero
    (relaxation.py:36-61).

    A device ``CSRMatrix`` gets a device tensor (computed by the library's kernel);
    anything else gets a host numpy array."""
    if isinstance(A, CSRMatrix):
        dt = torch.float64 if A.dtype == np.float64 else torch.float32
        out = torch.empty(A.shape[0], dtype=dt, device=A.device)
        N.call("amg_inverse_diagonal", A.desc(), 0 if dt == torch.float64 else 1, N.ptr(out), N.stream_ptr())
        return out
    d = matrix_diagonal(A)
    one = np.ones((), dtype=d.dtype)
    safe = np.where(d != 0, d, one)
    return np.where(d != 0, one / safe, np.zeros((), dtype=d.dtype))


def jacobi(A, x, b, Dinv, iterations=1, omega=1.0):
    """Damped Jacobi, ``iterations`` sweeps of
    ``x <- (1 - omega) x + omega (x + Dinv (b - A x))`` (relaxation.py:64-98).

    Returns a new tensor (the reference returns a new array too).  A may be a device
    ``CSRMatrix`` or anything convertible; x, b, Dinv are device tensors (host arrays are
    copied over and the result copied back)."""
    host = not isinstance(x, torch.Tensor) or not x.is_cuda
    A = CSRMatrix.from_any(A)
    dt = torch.float64 if A.dtype == np.float64 else torch.float32

    def dev(v):
        t = v if isinstance(v, torch.Tensor) else torch.as_tensor(np.asarray(v))
        return t.to(device=A.device, dtype=dt).contiguous()

    xd, bd, dd = dev(x), dev(b), dev(Dinv)
    k = 1 if xd.dim() == 1 else int(xd.shape[1])
    out = torch.empty_like(xd)
    N.call("amg_jacobi", A.desc(), 0 if dt == torch.float64 else 1, N.ptr(xd), N.ptr(bd), N.ptr(dd),
           N.ptr(out), k, int(iterations), float(omega), N.stream_ptr())
    if host:
        res = out.cpu()
        return res.numpy() if not isinstance(x, torch.Tensor) else res
    return out


def approximate_spectral_radius(A, Dinv, n_iter=15, seed=0, on_device=False):
    """Power-iteration estimate of rho(D^-1 A) (relaxation.py:101-132), on the host.

    ``on_device=True`` (A a CUDA ``CSRMatrix``) runs the same 15 steps from the same start
    vector with the library's SpMV kernel and device reductions: the result agrees with
    the host estimate to rounding (the norms sum in a different order), and no matrix is
    copied to the host, which matters for hierarchies assembled on the device."""
    if on_device:
        return _spectral_radius_device(A, Dinv, n_iter, seed)
    H = _host_csr(A)
    Dinv = np.asarray(Dinv.detach().cpu().numpy() if isinstance(Dinv, torch.Tensor) else Dinv)
    rng = np.random.default_rng(seed)
    v = np.asarray(rng.standard_normal(H.shape[0]), dtype=Dinv.dtype)
    v = v / np.linalg.norm(v)
    rho = 1.0
    for _ in range(n_iter):
        w = Dinv * (H @ v)
        rho = float(np.linalg.norm(w))
        if rho == 0.0:
            break
        v = w / rho
    return rho


def _spectral_radius_device(A, Dinv, n_iter, seed):
    if not isinstance(A, CSRMatrix) or A.device.type != "cuda":
        raise ValueError("on_device=True needs a CUDA CSRMatrix")
    dt = torch.float64 if A.val64 is not None else torch.float32
    d = torch.as_tensor(Dinv, device=A.device).to(dt)
    rng = np.random.default_rng(seed)
    v = torch.as_tensor(rng.standard_normal(A.shape[0]), device=A.device).to(dt)
    v = v / torch.linalg.vector_norm(v)
    rho = 1.0
    for _ in range(n_iter):
        w = d * A.matvec(v)
        rho = float(torch.linalg.vector_norm(w))
        if rho == 0.0:
            break
        v = w / rho
    return rho


def none(A, x, b):
    """Return x unchanged (no relaxation), relaxation.py:135-137."""
    return x
