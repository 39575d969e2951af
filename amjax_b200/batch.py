"""Many hierarchies in one launch: ``pcg_batch``.

The reference batches right-hand sides of ONE hierarchy with ``jax.vmap``
(README.md:60-66); independent systems of different sizes are separate calls.  Here
``pcg_batch`` hands every system (its own hierarchy and its own k right-hand sides) to the
library at once: one CUDA graph holds each system's CG loop as an independent branch with
its own device-side WHILE node, so a single launch solves all of them concurrently and the
GPU interleaves small and large systems.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _native as N


def pcg_batch(solvers, rhs, tol=1e-8, atol=0.0, maxiter=500, cycle="V", cycles_per_level=1,
              precision=None, return_info=False):
    """Solve ``solvers[i].A x_i = rhs[i]`` for every i (rhs[i]: [N_i] or [N_i, k_i]) with
    AMG-preconditioned CG, in one graph launch.  Returns the list of x_i (device tensors in
    the rhs's kind, like ``MultilevelSolver.pcg``), plus per-system info if asked."""
    if len(solvers) != len(rhs) or not solvers:
        raise ValueError("need one right-hand side per solver")
    if len({id(s) for s in solvers}) != len(solvers):
        raise ValueError("each solver may appear once per batch")
    if cycle not in ("V", "W", "F"):
        raise ValueError(f"Cycle {cycle!r} not supported. Use 'V', 'W', or 'F'.")
    precs = {s._precision(precision) for s in solvers}
    if len(precs) != 1:
        raise ValueError("all systems of a batch must run in one precision")
    prec = precs.pop()
    odt = torch.float32 if prec == N.PREC_F32 else torch.float64
    handles, bs, xs, backs, ks = [], [], [], [], []
    for s, b in zip(solvers, rhs):
        bd, back = s._rhs(b, odt)
        handles.append(s._native())
        bs.append(bd)
        xs.append(torch.empty_like(bd))
        backs.append(back)
        ks.append(1 if bd.dim() == 1 else int(bd.shape[1]))
    n = len(solvers)
    tot = sum(ks)
    iters = (C.c_int32 * tot)()
    rel = (C.c_double * tot)()
    H = (C.c_void_p * n)(*[h.value for h in handles])
    B = (C.c_void_p * n)(*[t.data_ptr() for t in bs])
    X = (C.c_void_p * n)(*[t.data_ptr() for t in xs])
    K = (C.c_int32 * n)(*ks)
    N.call("amg_pcg_batch", H, n, prec, B, X, K, float(tol), float(atol), int(maxiter), N.CYCLES[cycle],
           int(cycles_per_level), iters, rel, N.stream_ptr())
    out = [bk(x) for bk, x in zip(backs, xs)]
    if not return_info:
        return out
    info, off = [], 0
    for kk in ks:
        info.append({"iterations": list(iters[off:off + kk]), "relres": list(rel[off:off + kk])})
        off += kk
    return out, info
