"""Hand-written adjoint of the solve (amjax/multilevel.py:428-444) for torch.autograd.

Forward: x = solve(b, A) stores only the converged x (no iteration history).
Backward with upstream gradient v: lambda solves the ADJOINT system ``A^T lambda = v``
with the same kernels on the transposed hierarchy (the reference solves ``A lambda = v``,
correct only for symmetric A; for a symmetric hierarchy the two coincide and the
hierarchy is reused).  Then ``dL/db = lambda`` and ``dL/dA_ij = -sum_c lambda_ic x_jc``:
for a sparse operator (``SparseA``) sampled on A's stored pattern by the library's
kernel, for a dense tensor A the dense ``-lambda x^T`` the reference returns.  In FP64
and the mixed precisions the backward solve and the sampled product are one library call
(``amg_adjoint``, the entry point an XLA/JAX binding of the custom VJP would call).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp
import torch

from . import _native as N
from .csr import CSRMatrix


class SparseA:
    """A finest-level operator given as a fixed CSR pattern plus (differentiable) values
    in CSR order; pass it as ``A=`` to ``solve``/``pcg`` to get ``dL/dvalues``."""

    def __init__(self, pattern: CSRMatrix, values: torch.Tensor):
        if values.numel() != pattern.nnz:
            raise ValueError(f"expected {pattern.nnz} values, got {values.numel()}")
        self.pattern = pattern
        self.values = values
        self.shape = pattern.shape

    def csr(self) -> CSRMatrix:
        return self.pattern.with_values(self.values)

    def transposed_csr(self) -> CSRMatrix:
        perm, pat_t = _transpose_map(self.pattern)
        return pat_t.with_values(self.values.detach()[perm])


def _transpose_map(pattern: CSRMatrix):
    cached = getattr(pattern, "_tmap", None)
    if cached is not None:
        return cached
    H = pattern.to_scipy()
    idx = sp.csr_matrix((np.arange(H.nnz, dtype=np.float64) + 1.0, H.indices, H.indptr), shape=H.shape)
    T = idx.T.tocsr()
    T.sort_indices()
    perm = torch.as_tensor(T.data.astype(np.int64) - 1, device=pattern.device)
    pat_t = CSRMatrix.from_scipy(sp.csr_matrix((np.ones(T.nnz), T.indices, T.indptr), shape=T.shape),
                                 dtype=pattern.dtype, device=pattern.device)
    pattern._tmap = (perm, pat_t)
    return pattern._tmap


def needs_grad(b, A) -> bool:
    if not torch.is_grad_enabled():
        return False
    if isinstance(b, torch.Tensor) and b.requires_grad:
        return True
    if isinstance(A, torch.Tensor) and A.requires_grad:
        return True
    return isinstance(A, SparseA) and A.values.requires_grad


class _SolveFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, ml, opts, a_obj, b, a_tensor, x0):
        """x = x0 + A^-1 b, where b is already shifted to b - A x0 (x0 None: zero)."""
        del a_tensor  # carried only so autograd tracks it
        A0 = _forward_operator(ml, a_obj)
        x = _run(ml, opts, b.detach(), A0)
        if x0 is not None:
            x = x + x0
        ctx.ml, ctx.opts, ctx.a_obj = ml, opts, a_obj
        # dL/dA = -lambda x^T with the FULL solution x (the x0 term comes from b - A x0)
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, gx):
        (x,) = ctx.saved_tensors
        ml, opts, a_obj = ctx.ml, ctx.opts, ctx.a_obj
        mlt = ml.transposed()
        At = _transposed_operator(ml, a_obj)
        want_values = isinstance(a_obj, SparseA) and a_obj.values.requires_grad
        grad_a = None
        if ml._precision(opts["precision"]) != N.PREC_F32:  # one library call: A^-T solve + sampled product
            lam, gv = adjoint(mlt, opts, gx, x, At, a_obj.pattern if want_values else None)
            if want_values:
                grad_a = gv.to(a_obj.values.dtype)
        else:
            lam = _run(mlt, opts, gx.contiguous(), At)
            if want_values:
                grad_a = sampled_outer(a_obj.pattern, lam, x).to(a_obj.values.dtype)
        if isinstance(a_obj, torch.Tensor) and a_obj.requires_grad:
            lam2 = lam.reshape(lam.shape[0], -1)
            x2 = x.reshape(x.shape[0], -1)
            grad_a = (-(lam2 @ x2.T)).to(a_obj.dtype).to(a_obj.device)
        return None, None, None, lam, grad_a, None


def _forward_operator(ml, a_obj):
    if a_obj is None:
        return None
    if isinstance(a_obj, SparseA):
        return a_obj.csr()
    return ml._override(a_obj.detach() if isinstance(a_obj, torch.Tensor) else a_obj)


def _transposed_operator(ml, a_obj):
    if a_obj is None:
        return None
    if isinstance(a_obj, SparseA):
        return a_obj.transposed_csr()
    if isinstance(a_obj, torch.Tensor):
        return ml._override(a_obj.detach().T.contiguous())
    M = CSRMatrix.from_any(a_obj, dtype=ml.dtype)
    return CSRMatrix.from_scipy(M.to_scipy().T.tocsr(), dtype=ml.dtype, device=ml.levels[0].A.device)


def _run(ml, opts, bd, A0):
    prec = ml._precision(opts["precision"])
    odt = torch.float32 if prec == N.PREC_F32 else torch.float64
    bd = bd.to(device=ml.levels[0].A.device, dtype=odt).contiguous()
    if opts["method"] == "pcg":
        x, _ = ml._pcg_dev(bd, A0, opts["tol"], opts["atol"], opts["maxiter"], opts["cycle"],
                           opts["cycles_per_level"], prec)
    else:
        x, _ = ml._solve_dev(bd, A0, opts["tol"], opts["maxiter"], opts["cycle"], opts["cycles_per_level"], prec)
    return x


def adjoint(mlt, opts, gx, x, At=None, pattern=None):
    """The backward solve and the values gradient in one library call (``amg_adjoint``):
    ``lam = A^-T gx`` on the transposed hierarchy ``mlt`` (standalone cycles or PCG as
    ``opts["method"]`` says, the forward solve's tolerance, cycle and precision), and with
    ``pattern`` (A's CSR pattern) ``grad[e] = -sum_c lam[row(e), c] x[col(e), c]``.
    Returns ``(lam, grad or None)``; FP64 throughout."""
    dev = mlt.levels[0].A.device
    g = gx.detach().to(device=dev, dtype=torch.float64).contiguous()
    k = 1 if g.dim() == 1 else int(g.shape[1])
    lam = torch.empty_like(g)
    maxiter = opts["maxiter"] if opts["maxiter"] is not None else 10 * int(g.shape[0])
    grad = xd = None
    if pattern is not None:
        grad = torch.empty(pattern.nnz, dtype=torch.float64, device=dev)
        xd = x.detach().to(device=dev, dtype=torch.float64).contiguous()
    iters = (C.c_int32 * k)()
    rel = (C.c_double * k)()
    N.call("amg_adjoint", mlt._native(), mlt._precision(opts["precision"]), 1 if opts["method"] == "pcg" else 0,
           N.ptr(g), N.ptr(xd), k, float(opts["tol"]), float(opts["atol"]), int(maxiter), N.CYCLES[opts["cycle"]],
           int(opts["cycles_per_level"]), C.byref(At.desc()) if At is not None else None,
           C.byref(pattern.desc()) if pattern is not None else None, N.ptr(lam), N.ptr(grad), iters, rel,
           N.stream_ptr())
    mlt.last_info = {"iterations": list(iters), "relres": list(rel)}
    return lam, grad


def sampled_outer(pattern: CSRMatrix, lam: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
    """grad[e] = -sum_c lam[row(e), c] x[col(e), c] on the pattern (library kernel)."""
    lam = lam.to(torch.float64).contiguous()
    x = x.to(torch.float64).contiguous()
    k = 1 if lam.dim() == 1 else int(lam.shape[1])
    out = torch.empty(pattern.nnz, dtype=torch.float64, device=pattern.device)
    N.call("amg_sampled_outer", pattern.desc(), N.ptr(lam), N.ptr(x), k, N.ptr(out), N.stream_ptr())
    return out


def solve_with_grad(ml, b, A=None, x0=None, tol=1e-5, maxiter=100, cycle="V", cycles_per_level=1,
                    precision=None, return_info=False, method="solve", atol=0.0):
    """Differentiable ``solve`` / ``pcg`` (x0 is treated as a constant).  With x0 the
    solve runs on b - A x0 and adds x0 back; the gradient with respect to A still uses
    the full solution, as differentiating b - A x0 through the reference gives."""
    if method == "pcg" and maxiter is None:
        maxiter = 10 * ml.levels[0].A.shape[0]
    opts = dict(tol=tol, atol=atol, maxiter=maxiter, cycle=cycle, cycles_per_level=cycles_per_level,
                precision=precision, method=method)
    prec = ml._precision(precision)
    odt = torch.float32 if prec == N.PREC_F32 else torch.float64
    dev = ml.levels[0].A.device
    if not isinstance(b, torch.Tensor):
        b = torch.as_tensor(np.asarray(b))
    bt = b.to(device=dev, dtype=odt)
    a_tensor = A.values if isinstance(A, SparseA) else (A if isinstance(A, torch.Tensor) else None)
    if x0 is not None:
        x0t = torch.as_tensor(x0).to(device=dev, dtype=odt).detach()
        A0 = _forward_operator(ml, A)
        Aop = A0 if A0 is not None else ml.levels[0].A
        bt = bt - Aop.matvec(x0t)
    x = _SolveFn.apply(ml, opts, A, bt, a_tensor, x0t if x0 is not None else None)
    info = ml.last_info
    return (x, info) if return_info else x
