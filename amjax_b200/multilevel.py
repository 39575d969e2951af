"""``MultilevelSolver``: AMJax's solve-phase API over the B200 kernels.

Mirrors amjax/multilevel.py: ``from_pyamg`` (:125-186), ``solve`` (:341-394),
``aspreconditioner`` (:265-288), the level container (:16-58), complexities and
``__repr__`` (:188-263), ``coarse_grid_solver`` and its error rules (:448-536) and the
deprecated alias (:730-743).  The hierarchy's CSR arrays are uploaded once into torch
CUDA tensors; ``solve`` / ``pcg`` / the preconditioner each run as one CUDA-graph
launch of the library's fused kernels (``libamg_b200.so``).  There is no CPU path.

Extensions over the reference, all optional: ``precision`` ('f64' | 'f32' | 'mixed' |
'mixed-f64cg'; 'mixed': FP32 cycle inside FP64 refinement for ``solve``, and for ``pcg``
an FP32 CG whose FP64 solution and FP64 true residual are refreshed whenever the FP32
residual has dropped by a fixed factor and before a column stops; 'mixed-f64cg': the FP32
cycle inside an FP64 CG), right-hand sides stored ``[N, k]`` (k
columns solved at once, each freezing when converged as ``jax.vmap`` over the solve
does), ``pcg`` (the fused equivalent of ``jax.scipy.sparse.linalg.cg(A, b,
M=ml.aspreconditioner())``), ``return_info`` (iterations and final relative residual
per column).
"""

from __future__ import annotations

import ctypes as C
from warnings import warn

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
import torch

from . import _native as N
from .csr import CSRMatrix
from .relaxation import relaxation
from .relaxation import smoothing

__all__ = ["MultilevelSolver", "multilevel_solver", "coarse_grid_solver", "_NOT_IMPLEMENTED_SOLVERS"]

_PRECISIONS = {"f64": N.PREC_F64, "f32": N.PREC_F32, "mixed": N.PREC_MIXED,
               "mixed-f64cg": N.PREC_MIXED_F64CG}


class _Level:
    """One level (multilevel.py:16-58): ``A``, ``Dinv``, ``P``, ``R``, smoothers, and on
    the coarsest level the coarse-solver data (``A_inv``, ``lu_factor``/``piv``,
    ``Q``/``R_mat``, ``A_dense``)."""

    def __init__(self):
        self.A = None
        self.Dinv = None
        self.Dinv32 = None
        self.A_inv = None
        self.A_dense = None
        self.lu_factor = None
        self.piv = None
        self.Q = None
        self.R_mat = None
        self.P = None
        self.R = None
        self.presmoother = None
        self.postsmoother = None
        self._presmoother_spec = None
        self._postsmoother_spec = None


def _torch_dtype(dtype):
    return torch.float64 if np.dtype(dtype) == np.float64 else torch.float32


def _nnz(A):
    if hasattr(A, "nnz"):
        return int(A.nnz)
    if hasattr(A, "nse"):
        return int(A.nse)
    raise TypeError(f"Cannot determine nnz for type {type(A)}")


class MultilevelSolver:
    """Algebraic multigrid solve phase on B200 (see the module docstring)."""

    Level = _Level

    def __init__(self, levels, coarse_solver_fn=None, coarse_solver_name="pinv", coarse_solver_kwargs=None):
        self.levels = levels
        self.coarse_solver = coarse_solver_fn
        self._coarse_solver_name = coarse_solver_name
        self._coarse_solver_kwargs = coarse_solver_kwargs or {}
        self.symmetric_smoothing = False
        self._handle = None
        self._handle_key = None
        self._transposed = None
        self.last_info = None
        for lvl in self.levels[:-1]:
            if getattr(lvl, "R", None) is None and getattr(lvl, "P", None) is not None:
                lvl.R = lvl.P.T

    # ------------------------------------------------------------------ construction
    @classmethod
    def from_pyamg(cls, pyamg_solver, presmoother=("jacobi", {"iterations": 1, "omega": 1.0}),
                   postsmoother=("jacobi", {"iterations": 1, "omega": 1.0}), coarse_solver="pinv",
                   coarse_solver_kwargs=None, dtype=None, device=None):
        """Upload a PyAMG-shaped hierarchy (``.levels[i].A/.P/.R`` scipy matrices) once to
        the device and set up smoothers and the coarse solver (multilevel.py:125-186).

        The coarse pseudo-inverse / LU / QR are formed on the host in FP64 and stored in
        the hierarchy dtype (plus an FP32 copy for the mixed-precision cycle)."""
        if coarse_solver_kwargs is None:
            coarse_solver_kwargs = {}
        levels = _convert_hierarchy(pyamg_solver, dtype=dtype, device=device)
        coarse = levels[-1]
        if coarse_solver in ("pinv", "lu", "qr"):
            _setup_dense_coarse(coarse, coarse_solver, coarse_solver_kwargs)
        coarse_fn = coarse_grid_solver(coarse_solver, coarse, **coarse_solver_kwargs)
        ml = cls(levels, coarse_fn, coarse_solver_name=coarse_solver, coarse_solver_kwargs=coarse_solver_kwargs)
        smoothing.change_smoothers(ml, presmoother, postsmoother)
        return ml

    # ------------------------------------------------------------------ reporting
    def __repr__(self):
        total_nnz = sum(_nnz(lvl.A) for lvl in self.levels)
        out = "MultilevelSolver\n"
        out += f"Number of Levels: {len(self.levels)}\n"
        out += f"Operator Complexity: {self.operator_complexity():6.3f}\n"
        out += f"Grid Complexity: {self.grid_complexity():6.3f}\n"
        out += f"Cycle Complexity: {self.cycle_complexity():6.3f}\n"
        out += f"Coarse Solver: {self._coarse_solver_name!r}\n"
        out += "level unknowns nonzeros\n"
        for i, lvl in enumerate(self.levels):
            nnz = _nnz(lvl.A)
            out += f"{i:>6} {lvl.A.shape[0]:>11} {nnz:>12} [{100 * nnz / total_nnz:2.2f}%]\n"
        return out

    def operator_complexity(self):
        """Total stored nonzeros over the finest level's (multilevel.py:204-214)."""
        nnz = [_nnz(lvl.A) for lvl in self.levels]
        return sum(nnz) / float(nnz[0])

    def grid_complexity(self):
        """Total unknowns over the finest level's (used by ``__repr__``)."""
        rows = [lvl.A.shape[0] for lvl in self.levels]
        return sum(rows) / float(rows[0])

    def cycle_complexity(self, cycle="V"):
        """Work of one cycle relative to a fine-level SpMV (multilevel.py:216-263)."""
        cycle = str(cycle).upper()
        nnz = [_nnz(lvl.A) for lvl in self.levels]
        L = len(self.levels)

        def V(l):
            if L == 1:
                return nnz[0]
            if l == L - 2:
                return 2 * nnz[l] + nnz[l + 1]
            return 2 * nnz[l] + V(l + 1)

        def W(l):
            if L == 1:
                return nnz[0]
            if l == L - 2:
                return 2 * nnz[l] + nnz[l + 1]
            return 2 * nnz[l] + 2 * W(l + 1)

        def F(l):
            if L == 1:
                return nnz[0]
            if l == L - 2:
                return 2 * nnz[l] + nnz[l + 1]
            return 2 * nnz[l] + F(l + 1) + V(l + 1)

        if cycle == "V":
            flops = V(0)
        elif cycle == "W":
            flops = W(0)
        elif cycle == "F":
            flops = F(0)
        else:
            raise NotImplementedError(f"Cycle complexity for {cycle!r} not implemented.")
        return float(flops) / float(nnz[0])

    # ------------------------------------------------------------------ native handle
    @property
    def dtype(self):
        return self.levels[0].A.dtype

    def _invalidate(self):
        if self._handle is not None:
            N.load().amg_hierarchy_destroy(self._handle)
        self._handle = None
        self._handle_key = None
        self._transposed = None

    def __del__(self):
        try:
            if self._handle is not None and N._lib is not None:
                N._lib.amg_hierarchy_destroy(self._handle)
        except Exception:
            pass

    @staticmethod
    def _smoother_spec(fn, where):
        spec = getattr(fn, "_amg_spec", None)
        if spec is None:
            raise TypeError(f"{where}: smoother {fn!r} has no native form; use change_smoothers with "
                            "'jacobi' or None")
        name, it, om = spec
        kind = N.SMOOTH_JACOBI if name == "jacobi" else N.SMOOTH_NONE
        return N.amg_smoother(kind, int(it), float(om))

    def _native(self):
        key = tuple((getattr(l.presmoother, "_amg_spec", None), getattr(l.postsmoother, "_amg_spec", None))
                    for l in self.levels[:-1]) + (self._coarse_solver_name, tuple(sorted(self._coarse_solver_kwargs.items())))
        if self._handle is not None and self._handle_key == key:
            return self._handle
        lib = N.load()
        if self._handle is not None:
            lib.amg_hierarchy_destroy(self._handle)
            self._handle = None
        descs, cd = self._native_descs()
        h = C.c_void_p()
        N.check(lib.amg_hierarchy_create(descs, len(descs), C.byref(cd), C.byref(h)))
        self._handle = h
        self._handle_key = key
        return h

    def _native_descs(self):
        """The C-ABI level and coarse-solver descriptors over this hierarchy's device arrays."""
        L = len(self.levels)
        if L < 2:
            raise ValueError("a single-level hierarchy has no multigrid cycle (AMJax's _cycle needs >= 2 levels)")
        descs = (N.amg_level_desc * L)()
        empty = N.amg_csr()
        for i, lvl in enumerate(self.levels):
            d = descs[i]
            d.A = lvl.A.desc()
            d.P = lvl.P.desc() if i < L - 1 else empty
            d.R = lvl.R.desc() if i < L - 1 else empty
            d.dinv64 = lvl.Dinv.data_ptr() if lvl.Dinv.dtype == torch.float64 else None
            d.dinv32 = lvl.Dinv32.data_ptr()
            if i < L - 1:
                d.pre = self._smoother_spec(lvl.presmoother, f"level {i} presmoother")
                d.post = self._smoother_spec(lvl.postsmoother, f"level {i} postsmoother")
        coarse = self.levels[-1]
        cd = N.amg_coarse_desc()
        name = self._coarse_solver_name
        cd.kind = N.COARSE_KINDS[name]
        cd.n = coarse.A.shape[0]
        cd.iterations = int(self._coarse_solver_kwargs.get("iterations", 10))
        cd.omega = float(self._coarse_solver_kwargs.get("omega", 1.0))
        nat = getattr(coarse, "_native_coarse", {})
        for slot in ("m0_64", "m0_32", "m1_64", "m1_32", "perm"):
            t = nat.get(slot)
            setattr(cd, slot, t.data_ptr() if t is not None else None)
        return descs, cd

    def _precision(self, precision):
        if precision is None:
            return N.PREC_F64 if self.dtype == np.float64 else N.PREC_F32
        p = _PRECISIONS.get(str(precision).lower())
        if p is None:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}, got {precision!r}")
        if p != N.PREC_F32 and self.dtype != np.float64:
            raise ValueError("an FP32 hierarchy only supports precision='f32'")
        return p

    # ------------------------------------------------------------------ I/O helpers
    def _rhs(self, b, dtype):
        """b -> contiguous device tensor [N] or [N, k]; returns (tensor, back) where back
        maps a device result to the caller's kind (device tensor, CPU tensor, numpy)."""
        n = self.levels[0].A.shape[0]
        dev = self.levels[0].A.device
        if isinstance(b, torch.Tensor):
            on_dev = b.is_cuda
            t = b.detach()
            if t.dim() > 1 and t.shape[0] != n:
                t = t.reshape(-1)
            if not on_dev:
                if t.dtype != dtype:
                    t = t.to(dtype)
                if not t.is_pinned():
                    t = t.pin_memory()
                t = t.to(dev, non_blocking=True)
            t = t.to(device=dev, dtype=dtype).contiguous()
            if t.dim() == 1 and t.numel() != n:
                raise ValueError(f"b has {t.numel()} entries, expected {n}")
            return t, (lambda x: x) if on_dev else (lambda x: x.cpu())
        arr = np.asarray(b)
        if arr.ndim > 1 and arr.shape[0] != n:
            arr = arr.ravel()
        if arr.shape[0] != n:
            raise ValueError(f"b has {arr.shape[0]} rows, expected {n}")
        host = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float64 if dtype == torch.float64 else np.float32))
        t = host.pin_memory().to(dev, non_blocking=True)
        return t, (lambda x: x.cpu().numpy())

    def _override(self, A):
        if A is None:
            return None
        from .autograd import SparseA
        if isinstance(A, SparseA):
            A = A.csr()
        M = CSRMatrix.from_any(A, dtype=self.dtype, device=self.levels[0].A.device)
        if M.shape != self.levels[0].A.shape:
            raise ValueError(f"A has shape {M.shape}, expected {self.levels[0].A.shape}")
        return M

    # ------------------------------------------------------------------ solve
    def solve(self, b, A=None, x0=None, tol=1e-5, maxiter=100, cycle="V", cycles_per_level=1,
              precision=None, return_info=False, out=None):
        """Solve A x = b by repeated cycles (multilevel.py:341-425).

        Stops per column when ``||b - A x|| < tol ||b||`` or after ``maxiter`` cycles
        (non-convergence is silent, as in the reference).  ``A`` replaces the finest
        operator for residuals and smoothing while the rest of the hierarchy stays
        fixed.  Differentiable through ``torch.autograd`` with respect to ``b`` and to
        ``A``'s values (see :mod:`amjax_b200.autograd`)."""
        if cycle not in ("V", "W", "F"):
            raise ValueError(f"Cycle {cycle!r} not supported. Use 'V', 'W', or 'F'.")
        from . import autograd as _ag
        if _ag.needs_grad(b, A):
            return _ag.solve_with_grad(self, b, A=A, x0=x0, tol=tol, maxiter=maxiter, cycle=cycle,
                                       cycles_per_level=cycles_per_level, precision=precision,
                                       return_info=return_info)
        prec = self._precision(precision)
        odt = torch.float32 if prec == N.PREC_F32 else torch.float64
        bd, back = self._rhs(b, odt)
        A0 = self._override(A)
        if x0 is not None:
            x0d, _ = self._rhs(x0, odt)
            bd = bd - (A0 if A0 is not None else self.levels[0].A).matvec(x0d)
        x, info = self._solve_dev(bd, A0, tol, maxiter, cycle, cycles_per_level, prec)
        if x0 is not None:
            x = x + x0d
        res = _deliver(x, back, out)
        return (res, info) if return_info else res

    def _solve_dev(self, bd, A0, tol, maxiter, cycle, cycles_per_level, prec):
        h = self._native()
        k = 1 if bd.dim() == 1 else int(bd.shape[1])
        x = torch.empty_like(bd)
        iters = (C.c_int32 * k)()
        rel = (C.c_double * k)()
        N.call("amg_solve", h, prec, N.ptr(bd), N.ptr(x), k, float(tol), int(maxiter), N.CYCLES[cycle],
               int(cycles_per_level), C.byref(A0.desc()) if A0 is not None else None, iters, rel, N.stream_ptr())
        info = {"iterations": list(iters), "relres": list(rel)}
        self.last_info = info
        return x, info

    def pcg(self, b, A=None, x0=None, tol=1e-5, atol=0.0, maxiter=None, cycle="V", cycles_per_level=1,
            precision=None, return_info=False, out=None):
        """CG preconditioned by one cycle, fused on the device: the same iteration as
        ``jax.scipy.sparse.linalg.cg(A, b, M=ml.aspreconditioner(cycle))`` (stop when
        ``<r,r> <= max(tol^2 <b,b>, atol^2)``, default ``maxiter = 10 N``)."""
        if cycle not in ("V", "W", "F"):
            raise ValueError(f"Cycle {cycle!r} not supported. Use 'V', 'W', or 'F'.")
        from . import autograd as _ag
        if _ag.needs_grad(b, A):
            return _ag.solve_with_grad(self, b, A=A, x0=x0, tol=tol, maxiter=maxiter, cycle=cycle,
                                       cycles_per_level=cycles_per_level, precision=precision,
                                       return_info=return_info, method="pcg", atol=atol)
        prec = self._precision(precision)
        odt = torch.float32 if prec == N.PREC_F32 else torch.float64
        if A is None and x0 is None and prec != N.PREC_F32 and _host_block(b, self.levels[0].A.shape[0]):
            res, info = self._pcg_host(b, out, tol, atol, maxiter, cycle, cycles_per_level, prec)
            return (res, info) if return_info else res
        bd, back = self._rhs(b, odt)
        A0 = self._override(A)
        if x0 is not None:
            x0d, _ = self._rhs(x0, odt)
            bd = bd - (A0 if A0 is not None else self.levels[0].A).matvec(x0d)
        x, info = self._pcg_dev(bd, A0, tol, atol, maxiter, cycle, cycles_per_level, prec)
        if x0 is not None:
            x = x + x0d
        res = _deliver(x, back, out)
        return (res, info) if return_info else res

    def _pcg_host(self, b, out, tol, atol, maxiter, cycle, cycles_per_level, prec):
        """PCG of a host [N, k] block through ``amg_pcg_host``: the columns are solved in two
        blocks and each block's copy to and from the device overlaps the other's solve.
        Pinned CPU tensors are used in place; other host inputs are staged through pinned
        memory.  Returns the caller's kind (numpy in, numpy out; CPU tensor in, CPU tensor out)
        or fills ``out``."""
        n = self.levels[0].A.shape[0]
        if isinstance(b, torch.Tensor):
            bh, kind = b.detach(), "torch"
            if bh.dtype != torch.float64 or not bh.is_contiguous():
                bh = bh.to(torch.float64).contiguous()
        else:
            bh, kind = torch.from_numpy(np.ascontiguousarray(np.asarray(b, dtype=np.float64))), "numpy"
        if not bh.is_pinned():
            bh = bh.pin_memory()
        k = int(bh.shape[1])
        direct = (isinstance(out, torch.Tensor) and not out.is_cuda and out.dtype == torch.float64
                  and out.is_contiguous() and out.numel() == n * k and out.is_pinned())
        xh = out if direct else torch.empty((n, k), dtype=torch.float64).pin_memory()
        if maxiter is None:
            maxiter = 10 * n
        iters = (C.c_int32 * k)()
        rel = (C.c_double * k)()
        blocks = _host_blocks(k)
        N.call("amg_pcg_host", self._native(), prec, N.ptr(bh), N.ptr(xh), k, blocks, float(tol), float(atol),
               int(maxiter), N.CYCLES[cycle], int(cycles_per_level), iters, rel, N.stream_ptr())
        info = {"iterations": list(iters), "relres": list(rel)}
        self.last_info = info
        if out is not None:
            if not direct:
                out.copy_(xh.reshape(out.shape))
            return out, info
        return (xh.numpy() if kind == "numpy" else xh), info

    def _pcg_dev(self, bd, A0, tol, atol, maxiter, cycle, cycles_per_level, prec):
        h = self._native()
        k = 1 if bd.dim() == 1 else int(bd.shape[1])
        if maxiter is None:
            maxiter = 10 * int(bd.shape[0])
        x = torch.empty_like(bd)
        iters = (C.c_int32 * k)()
        rel = (C.c_double * k)()
        N.call("amg_pcg", h, prec, N.ptr(bd), N.ptr(x), k, float(tol), float(atol), int(maxiter),
               N.CYCLES[cycle], int(cycles_per_level), C.byref(A0.desc()) if A0 is not None else None,
               iters, rel, N.stream_ptr())
        info = {"iterations": list(iters), "relres": list(rel)}
        self.last_info = info
        return x, info

    def aspreconditioner(self, cycle="V", cycles_per_level=1, precision=None):
        """``M(b)``: one cycle from the zero vector (multilevel.py:265-288).  The
        returned callable keeps b's dtype; with ``precision='mixed'`` the cycle itself
        runs in FP32."""
        if cycle not in ("V", "W", "F"):
            raise ValueError(f"Cycle {cycle!r} not supported. Use 'V', 'W', or 'F'.")
        prec = self._precision(precision)
        cdt = torch.float64 if prec == N.PREC_F64 else torch.float32

        def matvec(b):
            h = self._native()
            bd, back = self._rhs(b, cdt)
            k = 1 if bd.dim() == 1 else int(bd.shape[1])
            x = torch.empty_like(bd)
            N.call("amg_precondition", h, prec, N.ptr(bd), N.ptr(x), k, N.CYCLES[cycle], int(cycles_per_level),
                   N.stream_ptr())
            if isinstance(b, torch.Tensor) and b.dtype != x.dtype:
                x = x.to(b.dtype)
            return back(x)

        matvec._amg_owner = self
        matvec._amg_cycle = (cycle, cycles_per_level, precision)
        return matvec

    # ------------------------------------------------------------------ adjoint support
    def transposed(self):
        """The hierarchy of A^T (levels A_l^T, P' = R^T, R' = P^T, coarse data of A_c^T,
        same smoothers): what the adjoint solve A^T lambda = v runs on.  For a symmetric
        hierarchy (every A_l symmetric and R = P^T) this is ``self``."""
        if self._transposed is not None:
            return self._transposed
        if getattr(self, "_is_symmetric", None) is None:
            self._is_symmetric = _hierarchy_symmetric(self)
        if self._is_symmetric:
            self._transposed = self
            return self
        levels = []
        dev = self.levels[0].A.device
        L = len(self.levels)
        for i, lvl in enumerate(self.levels):
            t = _Level()
            t.A = CSRMatrix.from_scipy(lvl.A.to_scipy().T.tocsr(), dtype=self.dtype, device=dev)
            t.Dinv, t.Dinv32 = lvl.Dinv, lvl.Dinv32
            if i < L - 1:
                t.P = CSRMatrix.from_scipy(lvl.R.to_scipy().T.tocsr(), dtype=self.dtype, device=dev)
                t.R = CSRMatrix.from_scipy(lvl.P.to_scipy().T.tocsr(), dtype=self.dtype, device=dev)
                t.presmoother, t.postsmoother = lvl.presmoother, lvl.postsmoother
                t._presmoother_spec, t._postsmoother_spec = lvl._presmoother_spec, lvl._postsmoother_spec
            levels.append(t)
        coarse = levels[-1]
        if self._coarse_solver_name in ("pinv", "lu", "qr"):
            _setup_dense_coarse(coarse, self._coarse_solver_name, self._coarse_solver_kwargs)
        fn = coarse_grid_solver(self._coarse_solver_name, coarse, **self._coarse_solver_kwargs)
        mt = MultilevelSolver(levels, fn, self._coarse_solver_name, dict(self._coarse_solver_kwargs))
        mt.symmetric_smoothing = self.symmetric_smoothing
        mt._is_symmetric = False
        mt._transposed = self
        self._transposed = mt
        return mt


def _host_blocks(k) -> int:
    """Column blocks of a host-buffer PCG: 2 for k >= 16 (AMG_HOST_BLOCKS overrides)."""
    import os
    v = os.environ.get("AMG_HOST_BLOCKS")
    if v and v.isdigit() and int(v) >= 1:
        return min(int(v), k)
    return 2 if k >= 16 else 1


def _host_block(b, n) -> bool:
    """b is a host [n, k >= 2] block (numpy or a CPU tensor): the overlapped host path."""
    if isinstance(b, torch.Tensor):
        return (not b.is_cuda) and b.dim() == 2 and b.shape[0] == n and b.shape[1] >= 2
    if isinstance(b, np.ndarray):
        return b.ndim == 2 and b.shape[0] == n and b.shape[1] >= 2
    return False


def _deliver(x, back, out):
    """Return the device result in the caller's kind, or copy it into ``out`` (a
    preallocated tensor, e.g. pinned host memory: the copy is then asynchronous on the
    current stream and complete once that stream is synchronised)."""
    if out is None:
        return back(x)
    out.copy_(x.reshape(out.shape), non_blocking=True)
    return out


def _hierarchy_symmetric(ml) -> bool:
    for i, lvl in enumerate(ml.levels):
        A = lvl.A.to_scipy()
        if (A - A.T).count_nonzero() != 0:
            return False
        if i < len(ml.levels) - 1:
            P, R = lvl.P.to_scipy(), lvl.R.to_scipy()
            if P.shape != R.T.shape or (P - R.T).count_nonzero() != 0:
                return False
    return True


# ---------------------------------------------------------------------- hierarchy set-up

def _convert_hierarchy(pyamg_solver, dtype=None, device=None):
    """PyAMG levels -> device levels (multilevel.py:557-590).  dtype defaults to the
    finest A's; Dinv in that dtype (plus an FP32 copy); a missing R becomes P^T."""
    levels = []
    for py_lvl in pyamg_solver.levels:
        lvl = _Level()
        A_host = sp.csr_matrix(py_lvl.A)
        if dtype is None:
            dtype = A_host.dtype
        dtype = np.dtype(dtype)
        lvl.A = CSRMatrix.from_scipy(A_host, dtype=dtype, device=device)
        dinv = relaxation.inverse_diagonal(lvl.A.to_scipy())
        dev = lvl.A.device
        lvl.Dinv = torch.as_tensor(dinv).to(dev)
        lvl.Dinv32 = lvl.Dinv.to(torch.float32) if dtype == np.float64 else lvl.Dinv
        if getattr(py_lvl, "P", None) is not None:
            lvl.P = CSRMatrix.from_scipy(py_lvl.P, dtype=dtype, device=dev)
        if getattr(py_lvl, "R", None) is not None:
            lvl.R = CSRMatrix.from_scipy(py_lvl.R, dtype=dtype, device=dev)
        levels.append(lvl)
    for lvl in levels[:-1]:
        if lvl.R is None:
            lvl.R = CSRMatrix.from_scipy(lvl.P.to_scipy().T.conj().tocsr(), dtype=lvl.P.dtype, device=lvl.P.device)
    return levels


def _pinv_fp64(M, kwargs):
    """Pseudo-inverse in FP64 with JAX's default cut-off (max(m, n) * eps * sigma_max),
    or the caller's ``rtol`` / ``rcond`` (the reference calls jnp.linalg.pinv(A, **kw))."""
    U, s, Vt = np.linalg.svd(M, full_matrices=False)
    r = kwargs.get("rtol", kwargs.get("rcond"))
    if r is None:
        r = max(M.shape) * np.finfo(np.float64).eps
    cut = r * (s[0] if s.size else 0.0)
    sinv = np.where(s > cut, 1.0 / np.where(s > cut, s, 1.0), 0.0)
    return (Vt.T * sinv) @ U.T


def _setup_dense_coarse(coarse, name, kwargs):
    """Dense coarse data (multilevel.py:173-181), formed on the host in FP64."""
    dtype = coarse.A.dtype
    dev = coarse.A.device
    Ad64 = coarse.A.to_scipy().toarray().astype(np.float64)
    tdt = _torch_dtype(dtype)
    coarse.A_dense = torch.as_tensor(Ad64).to(device=dev, dtype=tdt)
    nat = {}

    def both(name_, M):
        M = np.ascontiguousarray(M)
        t = torch.as_tensor(M).to(device=dev, dtype=tdt)
        nat[name_ + "_64"] = t if tdt == torch.float64 else None
        nat[name_ + "_32"] = torch.as_tensor(M.astype(np.float32)).to(dev)
        return t

    if name == "pinv":
        coarse.A_inv = both("m0", _pinv_fp64(Ad64, kwargs))
    elif name == "lu":
        lu, piv = sla.lu_factor(Ad64)
        coarse.lu_factor = both("m0", lu)
        coarse.piv = torch.as_tensor(piv.astype(np.int32)).to(dev)
        perm = np.arange(len(piv))
        for i, p in enumerate(piv):
            perm[i], perm[p] = perm[p], perm[i]
        nat["perm"] = torch.as_tensor(perm.astype(np.int32)).to(dev)
    elif name == "qr":
        Q, R = np.linalg.qr(Ad64)
        coarse.Q = both("m0", Q)
        coarse.R_mat = both("m1", R)
    coarse._native_coarse = nat


_NOT_IMPLEMENTED_SOLVERS = {
    "cholesky", "pinv2", "splu", "cg", "gmres", "bicgstab",
    "bicg", "cgs", "qmr", "minres", "fgmres", "gauss_seidel",
    "sor", "block_jacobi", "block_gauss_seidel",
}


def coarse_grid_solver(solver_name, lvl, **kwargs):
    """A coarse-grid solver callable ``(A, x, b) -> x`` (multilevel.py:455-498).

    The native cycle applies the coarse solve inside its own graph; this callable is the
    reference's stand-alone form of the same operation (device tensors in and out)."""
    if solver_name in _NOT_IMPLEMENTED_SOLVERS:
        raise NotImplementedError(
            f"'{solver_name}' coarse solver is not yet implemented in AMJax. "
            f"Available: ['jacobi', 'pinv', 'lu', 'qr']")
    if solver_name == "jacobi":
        iterations = kwargs.get("iterations", 10)
        omega = kwargs.get("omega", 1.0)

        def solve(A, x, b):
            return relaxation.jacobi(A, x, b, lvl.Dinv, iterations=iterations, omega=omega)
    elif solver_name == "pinv":
        def solve(A, x, b):
            del A, x
            if getattr(lvl, "A_inv", None) is None:
                _setup_dense_coarse(lvl, "pinv", kwargs)
            return lvl.A_inv @ _dev_like(b, lvl.A_inv)
    elif solver_name == "lu":
        def solve(A, x, b):
            del A, x
            if getattr(lvl, "lu_factor", None) is None:
                _setup_dense_coarse(lvl, "lu", kwargs)
            LU = lvl.lu_factor
            bb = _dev_like(b, LU)[lvl._native_coarse["perm"].long()]
            y = torch.linalg.solve_triangular(LU, bb.reshape(len(bb), -1), upper=False, unitriangular=True)
            return torch.linalg.solve_triangular(LU, y, upper=True).reshape(bb.shape)
    elif solver_name == "qr":
        def solve(A, x, b):
            del A, x
            if getattr(lvl, "Q", None) is None:
                _setup_dense_coarse(lvl, "qr", kwargs)
            y = lvl.Q.T @ _dev_like(b, lvl.Q)
            return torch.linalg.solve_triangular(lvl.R_mat, y.reshape(len(y), -1), upper=True).reshape(y.shape)
    else:
        raise ValueError(f"Unknown coarse solver {solver_name!r}. Available: ['jacobi', 'pinv', 'lu', 'qr']")
    solve.__name__ = solver_name
    return solve


def _dev_like(b, ref):
    if not isinstance(b, torch.Tensor):
        b = torch.as_tensor(np.asarray(b))
    return b.to(device=ref.device, dtype=ref.dtype)


class multilevel_solver(MultilevelSolver):  # noqa: N801
    """Deprecated alias for MultilevelSolver (multilevel.py:730-743)."""

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        warn("multilevel_solver is deprecated. Use MultilevelSolver.", DeprecationWarning, stacklevel=2)
