"""Algorithmic byte model of the solve phase (used for achieved-bandwidth figures).

A fixed model of the bytes each operation must move at least once, independent of how
the kernels fuse them (so the GB/s figure is comparable across implementations):

* matrix pass ``M(s) = nnz (s + 4) + 4 (rows + 1)`` (values + int32 columns + row
  pointers);
* Jacobi sweep on level l: ``M_A + k s 3 N_l + s N_l`` (read x, b, write x; Dinv once);
* residual + restriction: ``M_A + M_R + k s (2 N_l + N_{l+1})``;
* prolongation + correction: ``M_P + k s (2 N_l + N_{l+1})``;
* coarse solve: ``s n_c^2 + 2 k s n_c``;
* outer standalone trip (FP64): ``M_A(8) + 8 k 3 N`` (residual + norm; refinement
  update folded in);
* outer CG step (outer precision): ``M_A(so) + so k 9 N`` (p, q, x, r, z each read or
  written once: q = A p; x, r updates; p update).

``s`` is the cycle's value size (8 FP64, 4 FP32), ``so`` the outer loop's.
"""

from __future__ import annotations


def _mpass(nnz, rows, s):
    return nnz * (s + 4) + 4 * (rows + 1)


def cycle_bytes(levels, k, s, cycle="V", cycles_per_level=1, pre_iters=1, post_iters=1):
    """Bytes of one cycle.  ``levels``: list of dicts with n, nnz_A, nnz_P, nnz_R."""
    L = len(levels)

    def visit(l, ct):
        lv = levels[l]
        n, nc = lv["n"], levels[l + 1]["n"]
        MA = _mpass(lv["nnz_A"], n, s)
        b = (pre_iters + post_iters) * (MA + k * s * 3 * n + s * n)
        b += MA + _mpass(lv["nnz_R"], nc, s) + k * s * (2 * n + nc)
        b += _mpass(lv["nnz_P"], n, s) + k * s * (2 * n + nc)
        if l == L - 2:
            b += s * nc * nc + 2 * k * s * nc
        elif ct == "V":
            b += visit(l + 1, "V")
        elif ct == "W":
            b += 2 * visit(l + 1, "W")
        else:
            b += visit(l + 1, "F") + cycles_per_level * visit(l + 1, "V")
        return b

    return visit(0, cycle)


def solve_bytes(levels, k, iterations, method="pcg", cycle_s=8, outer_s=8, **kw):
    """Bytes of a whole solve: ``iterations`` outer trips plus the set-up pass."""
    n = levels[0]["n"]
    c = cycle_bytes(levels, k, cycle_s, **kw)
    if method == "pcg":
        step = _mpass(levels[0]["nnz_A"], n, outer_s) + outer_s * k * 9 * n + c
        setup = outer_s * k * 3 * n + c
    else:
        step = _mpass(levels[0]["nnz_A"], n, 8) + 8 * k * 3 * n + c
        setup = 8 * k * 2 * n
    return setup + iterations * step


def jacobi_sweep_bytes(n, nnz, k, s):
    """One Jacobi sweep (the dominant kernel class)."""
    return _mpass(nnz, n, s) + k * s * 3 * n + s * n


def level_stats(ml):
    """Per-level sizes of a MultilevelSolver for the model."""
    out = []
    for i, lvl in enumerate(ml.levels):
        d = {"n": lvl.A.shape[0], "nnz_A": lvl.A.nnz}
        if i < len(ml.levels) - 1:
            d["nnz_P"] = lvl.P.nnz
            d["nnz_R"] = lvl.R.nnz
        out.append(d)
    return out
