"""``cg``: the Krylov driver the reference's users pair with ``aspreconditioner``.

The reference delegates to ``jax.scipy.sparse.linalg.cg(A, b, M=ml.aspreconditioner())``
(README.md:57, benchmarks/benchmark.ipynb cell 7).  ``cg`` here keeps that call shape:
when ``M`` is a preconditioner made by a ``MultilevelSolver`` and ``A`` is that solver's
finest operator (or a same-shape override), the whole iteration runs fused on the
device (``MultilevelSolver.pcg``); otherwise it raises, since there is no generic path.
Returns ``(x, info)`` like JAX (``info`` is the per-column iteration count and final
recursive relative residual, where JAX returns None).
"""

from __future__ import annotations

from .csr import CSRMatrix


def cg(A, b, x0=None, *, tol=1e-5, atol=0.0, maxiter=None, M=None):
    owner = getattr(M, "_amg_owner", None)
    if owner is None:
        raise TypeError("amjax_b200.cg needs M = MultilevelSolver.aspreconditioner(...)")
    cycle, cpl, precision = M._amg_cycle
    A0 = None
    if A is not None and A is not owner.levels[0].A:
        A0 = A if not isinstance(A, CSRMatrix) else A
    x, info = owner.pcg(b, A=A0, x0=x0, tol=tol, atol=atol, maxiter=maxiter, cycle=cycle,
                        cycles_per_level=cpl, precision=precision, return_info=True)
    return x, info
