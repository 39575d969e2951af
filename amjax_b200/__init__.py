"""amjax_b200: AMJax's multigrid solve phase on NVIDIA B200 (sm_100a).

Drop-in for ``amjax``'s public API (amjax/__init__.py:1-10): ``MultilevelSolver``,
``change_smoothers``, ``jacobi``, ``inverse_diagonal``.  The solve, the preconditioner,
the fused PCG and the adjoint run in hand-written CUDA kernels (``libamg_b200.so``,
C ABI in include/amg_b200.h) on the device; hierarchy set-up stays on the host.
"""

from .multilevel import MultilevelSolver, multilevel_solver, coarse_grid_solver
from .relaxation.smoothing import change_smoothers
from .relaxation.relaxation import jacobi, inverse_diagonal
from .csr import CSRMatrix
from .autograd import SparseA
from .krylov import cg
from .batch import pcg_batch

__all__ = [
    "MultilevelSolver",
    "change_smoothers",
    "jacobi",
    "inverse_diagonal",
    "CSRMatrix",
    "SparseA",
    "cg",
    "pcg_batch",
    "multilevel_solver",
    "coarse_grid_solver",
]
