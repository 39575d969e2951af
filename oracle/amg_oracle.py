"""CPU oracle: an FP64 numpy/scipy restatement of AMJax's multigrid solve phase.

TEST INFRASTRUCTURE ONLY.  Nothing in the shipped package imports this module; only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm
may call it, and there only as the checker or the timed CPU baseline.

Every function restates the reference file:line it cites (paths relative to the AMJax
project root).  Pinning: the reference itself (JAX + PyAMG) is not importable on these
machines, so the oracle is pinned against the known-answer tests the reference's own
test-suite holds (tests/relaxation/test_relaxation.py:42-101,
tests/test_multilevel.py:16-48,110-153,450-478) and against the convergence and
finite-difference properties of tests/test_multilevel.py:50-108,155-247; per-iterate
values of AMJax itself are not available here ("per-iterate parity unpinned").
"""

from __future__ import annotations

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

CYCLES = ("V", "W", "F")


# --------------------------------------------------------------------------- relaxation

def inverse_diagonal(A):
    """1/diag(A), zero where the diagonal is zero (amjax/relaxation/relaxation.py:36-61).

    The diagonal is the sum of the stored entries with row == col
    (relaxation.py:9-15, a scatter-add, so duplicates add up)."""
    A = sp.coo_matrix(A) if sp.issparse(A) else sp.coo_matrix(np.asarray(A))
    m = A.row == A.col
    d = np.zeros(A.shape[0], dtype=A.dtype)
    np.add.at(d, A.row[m], A.data[m])
    safe = np.where(d != 0, d, np.ones((), d.dtype))
    return np.where(d != 0, np.ones((), d.dtype) / safe, np.zeros((), d.dtype))


def jacobi(A, x, b, Dinv, iterations=1, omega=1.0):
    """Damped Jacobi (relaxation.py:64-98): per sweep ``temp = Dinv*(b - A@x) + x`` then
    ``x = (1 - omega)*x + omega*temp`` (relaxation.py:94-96), ``iterations`` times."""
    omega = np.asarray(omega, dtype=Dinv.dtype)
    for _ in range(int(iterations)):
        temp = Dinv * (b - A @ x) + x
        x = (1 - omega) * x + omega * temp
    return x


def approximate_spectral_radius(A, Dinv, n_iter=15, seed=0):
    """Power iteration on D^-1 A (relaxation.py:101-132): v0 ~ default_rng(seed) normal,
    normalised; rho = ||D^-1 A v|| after the last step, early exit when it hits 0."""
    rng = np.random.default_rng(seed)
    v = np.asarray(rng.standard_normal(A.shape[0]), dtype=Dinv.dtype)
    v = v / np.linalg.norm(v)
    rho = 1.0
    for _ in range(n_iter):
        w = Dinv * (A @ v)
        rho = float(np.linalg.norm(w))
        if rho == 0.0:
            break
        v = w / rho
    return rho


# --------------------------------------------------------------------------- smoothers

class Smoother:
    """Resolved smoother: ('jacobi', iterations, omega) or ('none', 0, 0)."""

    def __init__(self, name, iterations=1, omega=1.0):
        self.name, self.iterations, self.omega = name, int(iterations), float(omega)

    def __call__(self, A, x, b, Dinv):
        if self.name == "none":
            return x
        return jacobi(A, x, b, Dinv, self.iterations, self.omega)


def resolve_smoother(spec, A, Dinv):
    """Spec -> Smoother, following smoothing.py:85-99 (setup_jacobi, withrho => omega/rho)
    and smoothing.py:31-34,130-158 (None/'none' is the identity)."""
    name, kw = (spec if isinstance(spec, tuple) else (spec, {}))
    if name is None or name == "none":
        return Smoother("none")
    if name != "jacobi":
        raise ValueError(name)
    omega = kw.get("omega", 1.0)
    if kw.get("withrho", False):
        omega = omega / approximate_spectral_radius(A, Dinv)
    return Smoother("jacobi", kw.get("iterations", 1), omega)


def expand_specs(spec, n):
    """smoothing.py:45-56: a non-list spec is repeated; a short list repeats its last item."""
    specs = spec if isinstance(spec, list) else [spec]
    return (specs + [specs[-1]] * n)[:n]


# --------------------------------------------------------------------------- hierarchy

class Level:
    def __init__(self, A, P=None, R=None):
        self.A = sp.csr_matrix(A)
        self.P = None if P is None else sp.csr_matrix(P)
        self.R = None if R is None else sp.csr_matrix(R)
        if self.P is not None and self.R is None:
            self.R = sp.csr_matrix(self.P.T.conj())  # multilevel.py:586-588
        self.Dinv = inverse_diagonal(self.A)
        self.pre = self.post = None


class Hierarchy:
    """Oracle hierarchy: levels + resolved smoothers + coarse solver (multilevel.py:125-186)."""

    def __init__(self, mats, presmoother=("jacobi", {"iterations": 1, "omega": 1.0}),
                 postsmoother=("jacobi", {"iterations": 1, "omega": 1.0}),
                 coarse_solver="pinv", coarse_solver_kwargs=None, dtype=np.float64):
        self.levels = []
        for (A, P, R) in mats:
            self.levels.append(Level(A.astype(dtype), None if P is None else P.astype(dtype),
                                     None if R is None else R.astype(dtype)))
        n = len(self.levels) - 1
        pre = expand_specs(presmoother, max(n, 1))
        post = expand_specs(postsmoother, max(n, 1))
        for i in range(n):
            lvl = self.levels[i]
            lvl.pre = resolve_smoother(pre[i], lvl.A, lvl.Dinv)
            lvl.post = resolve_smoother(post[i], lvl.A, lvl.Dinv)
        self.coarse = CoarseSolver(coarse_solver, self.levels[-1], **(coarse_solver_kwargs or {}))

    @classmethod
    def from_host(cls, host, **kw):
        mats = [(l.A, getattr(l, "P", None), getattr(l, "R", None)) for l in host.levels]
        return cls(mats, **kw)

    def transposed(self):
        """Hierarchy of A^T: levels A_l^T with P' = R^T, R' = P^T, same smoothers and the
        transposed coarse operator (the adjoint solve needs A^T lambda = v)."""
        t = Hierarchy.__new__(Hierarchy)
        t.levels = []
        for lvl in self.levels:
            nl = Level(lvl.A.T.tocsr(), None if lvl.R is None else lvl.R.T.tocsr(),
                       None if lvl.P is None else lvl.P.T.tocsr())
            nl.pre, nl.post = lvl.pre, lvl.post
            t.levels.append(nl)
        t.coarse = CoarseSolver(self.coarse.name, t.levels[-1], **self.coarse.kwargs)
        return t


def pinv_jax_rule(M):
    """Pseudo-inverse with JAX's default cut-off rtol = max(m, n) * eps * sigma_max
    (the reference forms it with jnp.linalg.pinv, multilevel.py:177)."""
    U, s, Vt = np.linalg.svd(M, full_matrices=False)
    cut = max(M.shape) * np.finfo(M.dtype).eps * (s[0] if s.size else 0.0)
    sinv = np.where(s > cut, 1.0 / np.where(s > cut, s, 1.0), 0.0)
    return (Vt.T * sinv) @ U.T


class CoarseSolver:
    """multilevel.py:455-536: 'pinv' (A_inv @ b), 'lu', 'qr', 'jacobi' (10 sweeps, omega 1
    by default, from the zero vector the cycle passes in)."""

    def __init__(self, name, lvl, **kwargs):
        self.name, self.kwargs = name, dict(kwargs)
        Ad = lvl.A.toarray()
        self.Dinv = lvl.Dinv
        if name == "pinv":
            self.Ainv = pinv_jax_rule(Ad) if "rcond" not in kwargs else np.linalg.pinv(Ad, rcond=kwargs["rcond"])
        elif name == "lu":
            self.lu = sla.lu_factor(Ad)
        elif name == "qr":
            self.Q, self.Rm = np.linalg.qr(Ad)
        elif name == "jacobi":
            self.iterations = kwargs.get("iterations", 10)
            self.omega = kwargs.get("omega", 1.0)
        else:
            raise ValueError(name)

    def __call__(self, A, x, b):
        if self.name == "pinv":
            return self.Ainv @ b
        if self.name == "lu":
            return sla.lu_solve(self.lu, b)
        if self.name == "qr":
            return sla.solve_triangular(self.Rm, self.Q.T @ b)
        return jacobi(A, x, b, self.Dinv, self.iterations, self.omega)


# --------------------------------------------------------------------------- cycle / solve

def cycle(ml, x, b, cycle="V", cycles_per_level=1, A=None):
    """One multigrid cycle (multilevel.py:290-339), recursion included: pre-smooth,
    ``R @ (b - A x)``, coarse solve at level L-2 (once, also for W), V: one recursion,
    W: two, F: one F recursion then ``cycles_per_level`` V recursions; ``x + P @ e``;
    post-smooth.  ``A`` replaces the operator on level 0 only (line 318)."""
    if cycle not in CYCLES:
        raise ValueError(f"Cycle {cycle!r} not supported. Use 'V', 'W', or 'F'.")
    L = len(ml.levels)

    def rec(l, x, b, ct):
        lvl = ml.levels[l]
        Al = A if (l == 0 and A is not None) else lvl.A
        x = lvl.pre(Al, x, b, lvl.Dinv)
        cb = lvl.R @ (b - Al @ x)
        cx = np.zeros_like(cb)
        if l == L - 2:
            cx = ml.coarse(ml.levels[-1].A, cx, cb)
        elif ct == "V":
            cx = rec(l + 1, cx, cb, "V")
        elif ct == "W":
            cx = rec(l + 1, cx, cb, "W")
            cx = rec(l + 1, cx, cb, "W")
        elif ct == "F":
            cx = rec(l + 1, cx, cb, "F")
            for _ in range(cycles_per_level):
                cx = rec(l + 1, cx, cb, "V")
        x = x + lvl.P @ cx
        x = lvl.post(Al, x, b, lvl.Dinv)
        return x

    return rec(0, x, b, cycle)


def solve_loop(ml, b, tol=1e-5, maxiter=100, cycle_type="V", cycles_per_level=1, A=None, history=None):
    """multilevel.py:407-425: x0 = 0, normb = ||b|| (0 -> 1), loop while
    ``it < maxiter and ||b - A x|| >= tol * normb``.  Returns (x, iterations, relres).
    If ``history`` is a list, every iterate is appended to it."""
    A = ml.levels[0].A if A is None else A
    normb = np.linalg.norm(b)
    if normb == 0.0:
        normb = 1.0
    x = np.zeros_like(b)
    normr = np.linalg.norm(b - A @ x)
    it = 0
    while it < maxiter and normr >= tol * normb:
        x = cycle(ml, x, b, cycle_type, cycles_per_level, A=A if A is not ml.levels[0].A else None)
        normr = np.linalg.norm(b - A @ x)
        it += 1
        if history is not None:
            history.append(x.copy())
    return x, it, normr / normb


def solve(ml, b, A=None, x0=None, tol=1e-5, maxiter=100, cycle_type="V", cycles_per_level=1):
    """multilevel.py:341-394 (forward value only): optional x0 shift, then the loop."""
    b = np.ravel(np.asarray(b))
    if x0 is not None:
        x0 = np.ravel(np.asarray(x0))
        b = b - (ml.levels[0].A if A is None else A) @ x0
    x, it, rr = solve_loop(ml, b, tol, maxiter, cycle_type, cycles_per_level, A=A)
    if x0 is not None:
        x = x + x0
    return x, it


def aspreconditioner(ml, cycle_type="V", cycles_per_level=1):
    """multilevel.py:265-288: M(b) = one cycle from the zero vector."""
    return lambda b: cycle(ml, np.zeros_like(b), b, cycle_type, cycles_per_level)


def cg(A, b, x0=None, tol=1e-5, atol=0.0, maxiter=None, M=None, history=None):
    """Preconditioned CG with jax.scipy.sparse.linalg.cg's semantics (the reference's
    Krylov driver, benchmarks/benchmark.ipynb cell 7, README.md:57): stop when
    ``<r, r> <= max(tol^2 <b, b>, atol^2)`` or after ``maxiter`` steps, recursive
    residual, default ``maxiter = 10 * len(b)``.  Returns (x, iterations)."""
    Aop = (lambda v: A @ v) if not callable(A) else A
    M = (lambda v: v) if M is None else M
    maxiter = 10 * b.shape[0] if maxiter is None else maxiter
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=b.dtype)
    bs = float(b @ b)
    atol2 = max(tol * tol * bs, atol * atol)
    r = b - Aop(x)
    z = M(r)
    p = z
    gamma = float(r @ z)
    k = 0
    while float(r @ r) > atol2 and k < maxiter:
        Ap = Aop(p)
        alpha = gamma / float(p @ Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        z = M(r)
        gamma_new = float(r @ z)
        beta = gamma_new / gamma
        p = z + beta * p
        gamma = gamma_new
        k += 1
        if history is not None:
            history.append(x.copy())
    return x, k


# --------------------------------------------------------------------------- adjoint

def adjoint(ml, x, v, tol=1e-10, maxiter=100, cycle_type="V", cycles_per_level=1, A=None, transpose=True):
    """Backward of solve (multilevel.py:438-442): lambda solves the adjoint system, the
    gradient is grad_b = lambda, grad_A = -lambda x^T.  The reference solves A lambda = v
    (correct only for symmetric A); with ``transpose=True`` the oracle solves
    A^T lambda = v on the transposed hierarchy.  Returns (lambda, dense grad_A)."""
    if transpose:
        mlt = ml.transposed()
        At = None if A is None else sp.csr_matrix(A).T.tocsr()
        lam, _, _ = solve_loop(mlt, v, tol, maxiter, cycle_type, cycles_per_level, A=At)
    else:
        lam, _, _ = solve_loop(ml, v, tol, maxiter, cycle_type, cycles_per_level, A=A)
    return lam, -np.outer(lam, x)


def sampled_grad(A, lam, x):
    """-sum_c lam[i, c] x[j, c] on A's stored pattern (CSR order) for [N] or [N, k] inputs."""
    A = sp.csr_matrix(A)
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    lam2 = lam.reshape(A.shape[0], -1)
    x2 = x.reshape(A.shape[1], -1)
    return -np.einsum("ij,ij->i", lam2[rows], x2[A.indices])


# --------------------------------------------------------------------------- complexities

def cycle_complexity(nnz, cycle="V"):
    """multilevel.py:216-263 on a list of per-level nnz."""
    cycle = str(cycle).upper()
    L = len(nnz)

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
        f = V(0)
    elif cycle == "W":
        f = W(0)
    elif cycle == "F":
        f = F(0)
    else:
        raise NotImplementedError(f"Cycle complexity for {cycle!r} not implemented.")
    return float(f) / float(nnz[0])
