"""Host-side AMG hierarchy construction, standing in for PyAMG's solver factories.

The reference never builds a hierarchy itself: ``MultilevelSolver.from_pyamg``
(amjax/multilevel.py:125-186) converts one made by ``pyamg.smoothed_aggregation_solver``
or ``pyamg.ruge_stuben_solver`` (benchmarks/benchmark.ipynb cell 5,
tests/test_multilevel.py:59,82).  PyAMG (``pyamg>=4.0.0``, unpinned in
pyproject.toml:32) is not importable on these machines, so this module restates the
published setup algorithms in numpy/scipy and returns an object with PyAMG's shape:
``.levels[i].A`` (scipy CSR), ``.levels[i].P`` / ``.levels[i].R`` on every level but
the coarsest.  ``from_pyamg`` accepts either this object or a real PyAMG one.

Algorithms (restated from the literature, not from PyAMG's source):

* Smoothed aggregation (Vanek, Mandel & Brezina, Computing 56, 1996) with PyAMG's
  documented defaults: symmetric strength with theta = 0, standard (greedy three-pass)
  aggregation, the constant candidate improved by 4 symmetric Gauss-Seidel sweeps on
  ``A b = 0`` at the finest level, tentative prolongator from a per-aggregate QR of the
  candidate, one damped-Jacobi prolongator smoothing step with ``omega = 4/3 / rho(D^-1 A)``,
  ``R = P^T`` and the Galerkin product ``A_c = R A P``; ``max_levels = 10``,
  ``max_coarse = 10``.
* Ruge-Stueben classical AMG (Ruge & Stueben, 1987): classical strength with
  ``theta = 0.25`` on ``|a_ij|``, the first-pass C/F splitting, direct interpolation,
  ``R = P^T``, Galerkin coarse operators.
* Root-node AMG (Manteuffel, Olson, Schroder & Southworth, SISC 39, 2017), with the
  energy-minimising prolongation of Olson, Schroder & Tuminaro (Num. Lin. Alg. Appl. 18,
  2011): standard aggregation with one root node per aggregate; a tentative prolongator
  that injects at the root nodes (``P[root_j, :] = e_j``) and reproduces the candidate
  (``P B_c = B``); then a few Jacobi-preconditioned CG iterations on ``trace(P^T A P)``
  over the sparsity pattern of ``A^degree T`` with both constraints kept (``degree = 2``,
  ``maxiter = 4``).
* Pairwise aggregation (Notay, ETNA 37, 2010): two passes of pairing each node with its
  most negatively coupled free neighbour among the strong ones (``a_ij < -beta max_k
  |a_ik|``, ``beta = 0.25``; strongly diagonally dominant rows stay out of the coarse
  grid), so aggregates hold at most four nodes; unsmoothed piecewise-constant
  prolongator, ``R = P^T``.

The resulting arrays are NOT bit-identical to PyAMG's (tie-breaking and the spectral
radius estimate differ); the solve phase only needs some valid hierarchy, and the GPU
path and the oracle always consume the same arrays.
"""

from __future__ import annotations

import heapq

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

__all__ = [
    "HostLevel",
    "HostHierarchy",
    "smoothed_aggregation_solver",
    "ruge_stuben_solver",
    "air_solver",
    "rootnode_solver",
    "pairwise_solver",
    "save_hierarchy",
    "load_hierarchy",
]


class HostLevel:
    """One level of a host hierarchy: ``A`` and, except on the coarsest, ``P`` and ``R``."""

    def __init__(self, A, P=None, R=None):
        self.A = A
        if P is not None:
            self.P = P
        if R is not None:
            self.R = R


class HostHierarchy:
    """PyAMG-shaped container: ``levels`` is finest-first, scipy CSR throughout."""

    def __init__(self, levels, kind="unknown"):
        self.levels = levels
        self.kind = kind

    def __repr__(self):
        rows = ", ".join(f"{lvl.A.shape[0]}/{lvl.A.nnz}" for lvl in self.levels)
        return f"HostHierarchy({self.kind}: rows/nnz per level = {rows})"


def _csr(A):
    A = sp.csr_matrix(A)
    A.sum_duplicates()
    A.eliminate_zeros()
    A.sort_indices()
    return A


def _rho_dinv_a(A, steps=15):
    """Estimate of rho(D^-1 A) for the prolongator-smoothing weight.

    Symmetric A: ``steps`` Arnoldi (= Lanczos) steps on D^-1 A from a seeded random start,
    rho = the largest Ritz value (the short Krylov estimate the smoothed-aggregation
    literature uses; for a symmetric-similar operator Ritz values lie inside the spectrum).
    Nonsymmetric A: ARPACK, since Ritz values of a non-normal operator can overshoot.
    Exact eigenvalues for small matrices."""
    d = A.diagonal()
    dinv = np.where(d != 0, 1.0 / np.where(d != 0, d, 1.0), 0.0)
    n = A.shape[0]
    if n <= 64:
        return float(np.max(np.abs(np.linalg.eigvals((sp.diags(dinv) @ A).toarray()))))
    if (A != A.T).nnz != 0:
        DA = sp.diags(dinv) @ A
        try:
            v0 = np.random.default_rng(0).standard_normal(n)
            ev = spla.eigs(DA, k=1, which="LM", return_eigenvectors=False, v0=v0, tol=1e-4, maxiter=400)
            return float(np.abs(ev[0]))
        except Exception:
            pass
    m = min(steps, n)
    V = np.zeros((m + 1, n))
    H = np.zeros((m + 1, m))
    v = np.random.default_rng(0).standard_normal(n)
    V[0] = v / np.linalg.norm(v)
    for j in range(m):
        w = dinv * (A @ V[j])
        for i in range(j + 1):
            H[i, j] = w @ V[i]
            w = w - H[i, j] * V[i]
        H[j + 1, j] = np.linalg.norm(w)
        if H[j + 1, j] < 1e-14:
            m = j + 1
            break
        V[j + 1] = w / H[j + 1, j]
    return float(np.max(np.abs(np.linalg.eigvals(H[:m, :m]))))


# ---------------------------------------------------------------- smoothed aggregation

def _symmetric_strength(A, theta=0.0):
    """Keep off-diagonal a_ij with |a_ij| >= theta * sqrt(|a_ii a_jj|) (theta=0 keeps all)."""
    A = A.tocoo()
    off = A.row != A.col
    d = np.abs(_csr(A).diagonal())
    keep = off & (np.abs(A.data) >= theta * np.sqrt(d[A.row] * d[A.col]))
    S = sp.csr_matrix((np.ones(keep.sum()), (A.row[keep], A.col[keep])), shape=A.shape)
    return _csr(S)


def _standard_aggregation(S, return_roots=False):
    """Greedy three-pass aggregation on the strength graph S (diagonal-free CSR).

    Pass 1: every node whose neighbours are all free becomes a root; it and its
    neighbours form an aggregate.  Pass 2: each still-free node joins the aggregate of
    an aggregated neighbour.  Pass 3: each node still free starts a new aggregate with
    its free neighbours (it is that aggregate's root).  Nodes without neighbours stay
    unaggregated (index -1).  Returns (agg index per node, number of aggregates), and
    with ``return_roots`` also the root node of every aggregate.
    """
    n = S.shape[0]
    ptr, idx = S.indptr, S.indices
    agg = np.full(n, -2, dtype=np.int64)  # -2 free, -1 isolated
    deg = np.diff(ptr)
    agg[deg == 0] = -1
    nagg = 0
    roots = []
    ptr_l = ptr.tolist(); idx_l = idx.tolist(); agg_l = agg.tolist()
    for i in range(n):
        if agg_l[i] != -2:
            continue
        nb = idx_l[ptr_l[i]:ptr_l[i + 1]]
        if all(agg_l[j] == -2 for j in nb):
            agg_l[i] = nagg
            for j in nb:
                agg_l[j] = nagg
            roots.append(i)
            nagg += 1
    pass2 = agg_l[:]
    for i in range(n):
        if agg_l[i] != -2:
            continue
        for j in idx_l[ptr_l[i]:ptr_l[i + 1]]:
            if agg_l[j] >= 0:
                pass2[i] = agg_l[j]
                break
    agg_l = pass2
    for i in range(n):
        if agg_l[i] != -2:
            continue
        agg_l[i] = nagg
        for j in idx_l[ptr_l[i]:ptr_l[i + 1]]:
            if agg_l[j] == -2:
                agg_l[j] = nagg
        roots.append(i)
        nagg += 1
    if return_roots:
        return np.asarray(agg_l, dtype=np.int64), nagg, np.asarray(roots, dtype=np.int64)
    return np.asarray(agg_l, dtype=np.int64), nagg


def _symmetric_gauss_seidel(A, x, b, iterations):
    """``iterations`` symmetric (forward then backward) point Gauss-Seidel sweeps."""
    L = sp.tril(A, 0, format="csr")
    U = sp.triu(A, 0, format="csr")
    Ls = sp.triu(A, 1, format="csr")
    Us = sp.tril(A, -1, format="csr")
    for _ in range(iterations):
        x = spla.spsolve_triangular(L, b - Ls @ x, lower=True)
        x = spla.spsolve_triangular(U, b - Us @ x, lower=False)
    return x


def _fit_candidates(agg, nagg, B):
    """Tentative prolongator T and coarse candidates from a per-aggregate QR of B (1 column)."""
    n = B.shape[0]
    member = agg >= 0
    rows = np.nonzero(member)[0]
    cols = agg[member]
    bvals = B[member, 0]
    norms = np.sqrt(np.bincount(cols, weights=bvals * bvals, minlength=nagg))
    safe = np.where(norms > 0, norms, 1.0)
    T = sp.csr_matrix((bvals / safe[cols], (rows, cols)), shape=(n, nagg))
    return _csr(T), norms.reshape(-1, 1)


def smoothed_aggregation_solver(A, B=None, max_levels=10, max_coarse=10, theta=0.0,
                                improve_iterations=4, omega=4.0 / 3.0, **_ignored):
    """Build an SA hierarchy with the defaults listed in the module docstring."""
    A = _csr(A).astype(np.float64)
    B = np.ones((A.shape[0], 1)) if B is None else np.asarray(B, dtype=np.float64).reshape(A.shape[0], -1)
    levels = [HostLevel(A)]
    while len(levels) < max_levels and levels[-1].A.shape[0] > max_coarse:
        A = levels[-1].A
        S = _symmetric_strength(A, theta)
        agg, nagg = _standard_aggregation(S)
        if nagg == 0 or nagg >= A.shape[0]:
            break
        if len(levels) == 1 and improve_iterations:
            B = _symmetric_gauss_seidel(A, B[:, 0].copy(), np.zeros(A.shape[0]), improve_iterations).reshape(-1, 1)
        T, Bc = _fit_candidates(agg, nagg, B)
        d = A.diagonal()
        dinv = np.where(d != 0, 1.0 / np.where(d != 0, d, 1.0), 0.0)
        w = omega / _rho_dinv_a(A)
        P = _csr(T - w * (sp.diags(dinv) @ (A @ T)))
        R = _csr(P.T)
        Ac = _csr(R @ A @ P)
        levels[-1].P = P
        levels[-1].R = R
        levels.append(HostLevel(Ac))
        B = Bc
    return HostHierarchy(levels, kind="smoothed_aggregation")


# ---------------------------------------------------------------- root node

def _rootnode_tentative(agg, nagg, roots, B):
    """Tentative prolongator that injects at the root nodes: T[i, agg_i] = B_i / B_root,
    so T[root_j, :] = e_j and T B_c = B on aggregated rows, with B_c = B at the roots."""
    n = B.shape[0]
    b = B[:, 0]
    broot = b[roots]
    broot = np.where(broot != 0, broot, 1.0)
    member = agg >= 0
    rows = np.nonzero(member)[0]
    cols = agg[member]
    T = sp.csr_matrix((b[member] / broot[cols], (rows, cols)), shape=(n, nagg))
    return _csr(T), broot.reshape(-1, 1)


def _energy_prolongation(A, T, Bc, roots, free_rows, degree=2, maxiter=4):
    """Energy-minimising prolongator (Olson, Schroder & Tuminaro 2011): CG on
    ``trace(P^T A P)`` from ``P = T`` over corrections D that keep (1) the sparsity pattern
    of ``A^degree T``, (2) the root rows fixed (D[roots, :] = 0), (3) the candidate,
    ``D B_c = 0`` row by row; Jacobi (D^-1) preconditioned, Frobenius inner products."""
    n = A.shape[0]
    Pat = abs(T).tocsr()
    for _ in range(degree):
        Pat = abs(A) @ Pat
    Pat = _csr(Pat + abs(T))
    Pat.data[:] = 1.0
    keep = np.zeros(n)
    keep[free_rows] = 1.0
    keep[roots] = 0.0
    Pat = _csr(sp.diags(keep) @ Pat)  # rows that may change
    Pat.data[:] = 1.0
    bc = Bc[:, 0]
    wrow = np.asarray(Pat @ (bc * bc)).ravel()
    wrow = np.where(wrow > 0, wrow, 1.0)
    PatB = _csr(Pat @ sp.diags(bc))

    def project(M):
        M = _csr(M.multiply(Pat))
        c = np.asarray(M @ bc).ravel() / wrow  # remove each row's component along B_c
        return _csr(M - sp.diags(c) @ PatB)

    d = A.diagonal()
    dinv = sp.diags(np.where(d != 0, 1.0 / np.where(d != 0, d, 1.0), 0.0))
    P = T.copy()
    R = project(-(A @ P))
    Z = project(dinv @ R)
    rz = R.multiply(Z).sum()
    Pd = Z
    for _ in range(maxiter):
        if not np.isfinite(rz) or rz <= 0:
            break
        AP = A @ Pd
        pap = Pd.multiply(AP).sum()
        if pap <= 0:
            break
        alpha = rz / pap
        P = _csr(P + alpha * Pd)
        R = _csr(R - alpha * project(AP))
        Z = project(dinv @ R)
        rz_new = R.multiply(Z).sum()
        Pd = _csr(Z + (rz_new / rz) * Pd)
        rz = rz_new
    P.eliminate_zeros()
    return _csr(P)


def rootnode_solver(A, B=None, max_levels=10, max_coarse=10, theta=0.0, improve_iterations=4, degree=2,
                    maxiter=4, **_ignored):
    """Build a root-node hierarchy with the defaults listed in the module docstring."""
    A = _csr(A).astype(np.float64)
    B = np.ones((A.shape[0], 1)) if B is None else np.asarray(B, dtype=np.float64).reshape(A.shape[0], -1)
    levels = [HostLevel(A)]
    while len(levels) < max_levels and levels[-1].A.shape[0] > max_coarse:
        A = levels[-1].A
        S = _symmetric_strength(A, theta)
        agg, nagg, roots = _standard_aggregation(S, return_roots=True)
        if nagg == 0 or nagg >= A.shape[0]:
            break
        if len(levels) == 1 and improve_iterations:
            B = _symmetric_gauss_seidel(A, B[:, 0].copy(), np.zeros(A.shape[0]), improve_iterations).reshape(-1, 1)
        T, Bc = _rootnode_tentative(agg, nagg, roots, B)
        P = _energy_prolongation(A, T, Bc, roots, np.nonzero(agg >= 0)[0], degree, maxiter)
        R = _csr(P.T)
        levels[-1].P = P
        levels[-1].R = R
        levels.append(HostLevel(_csr(R @ A @ P)))
        B = Bc
    return HostHierarchy(levels, kind="rootnode")


# ---------------------------------------------------------------- pairwise

def _pairwise_pass(A, beta=0.25, dd_factor=5.0):
    """One pairing pass (Notay 2010, Algorithm 4.1 with natural node order): every free node
    i is paired with the free j != i of most negative a_ij among its strong negative
    couplings (a_ij < -beta max_k |a_ik|), or left alone when it has none.  Rows with
    a_ii > dd_factor * sum_{j != i} |a_ij| are left out of the coarse grid.  Returns the
    aggregate index per node (-1: left out) and the number of aggregates."""
    n = A.shape[0]
    A = _csr(A)
    ptr, idx, val = A.indptr, A.indices, A.data
    diag = A.diagonal()
    offsum = np.asarray(abs(A).sum(axis=1)).ravel() - np.abs(diag)
    agg = np.full(n, -2, dtype=np.int64)
    agg[diag > dd_factor * offsum] = -1
    nagg = 0
    for i in range(n):
        if agg[i] != -2:
            continue
        s, e = ptr[i], ptr[i + 1]
        cols, vals = idx[s:e], val[s:e]
        off = cols != i
        cols, vals = cols[off], vals[off]
        best = -1
        if len(cols):
            bound = -beta * np.max(np.abs(vals))
            cand = (vals < bound) & (agg[cols] == -2)
            if np.any(cand):
                cc, cv = cols[cand], vals[cand]
                best = int(cc[np.lexsort((cc, cv))[0]])  # most negative, ties by column
        agg[i] = nagg
        if best >= 0:
            agg[best] = nagg
        nagg += 1
    return agg, nagg


def _piecewise_constant(agg, nagg):
    member = agg >= 0
    rows = np.nonzero(member)[0]
    return _csr(sp.csr_matrix((np.ones(len(rows)), (rows, agg[member])), shape=(len(agg), nagg)))


def pairwise_solver(A, max_levels=10, max_coarse=10, beta=0.25, matchings=2, **_ignored):
    """Build a pairwise-aggregation hierarchy with the defaults in the module docstring."""
    A = _csr(A).astype(np.float64)
    levels = [HostLevel(A)]
    while len(levels) < max_levels and levels[-1].A.shape[0] > max_coarse:
        A = levels[-1].A
        P = None
        Ak = A
        for _ in range(matchings):
            agg, nagg = _pairwise_pass(Ak, beta)
            Pk = _piecewise_constant(agg, nagg)
            P = Pk if P is None else _csr(P @ Pk)
            Ak = _csr(Pk.T @ Ak @ Pk)
            if nagg <= max_coarse:
                break
        if P.shape[1] == 0 or P.shape[1] >= A.shape[0]:
            break
        R = _csr(P.T)
        levels[-1].P = P
        levels[-1].R = R
        levels.append(HostLevel(_csr(R @ A @ P)))
    return HostHierarchy(levels, kind="pairwise")


# ---------------------------------------------------------------- Ruge-Stueben

def _classical_strength(A, theta=0.25):
    """j strongly influences i when |a_ij| >= theta * max_{k != i} |a_ik| (diagonal dropped)."""
    A = A.tocoo()
    off = A.row != A.col
    r, c, v = A.row[off], A.col[off], np.abs(A.data[off])
    rmax = np.zeros(A.shape[0])
    np.maximum.at(rmax, r, v)
    keep = v >= theta * rmax[r]
    return _csr(sp.csr_matrix((np.ones(keep.sum()), (r[keep], c[keep])), shape=A.shape))


def _rs_first_pass(S):
    """First-pass Ruge-Stueben C/F splitting.  Returns a bool array, True for C points."""
    n = S.shape[0]
    St = _csr(S.T)
    sp_ptr, sp_idx = S.indptr.tolist(), S.indices.tolist()
    st_ptr, st_idx = St.indptr.tolist(), St.indices.tolist()
    lam = np.diff(St.indptr).tolist()
    state = [0] * n  # 0 unassigned, 1 C, 2 F
    for i in range(n):
        if lam[i] == 0 and sp_ptr[i + 1] == sp_ptr[i]:
            state[i] = 2
    heap = [(-lam[i], i) for i in range(n) if state[i] == 0]
    heapq.heapify(heap)
    while heap:
        negl, i = heapq.heappop(heap)
        if state[i] != 0 or -negl != lam[i]:
            continue
        state[i] = 1
        for j in st_idx[st_ptr[i]:st_ptr[i + 1]]:
            if state[j] == 0:
                state[j] = 2
                for k in sp_idx[sp_ptr[j]:sp_ptr[j + 1]]:
                    if state[k] == 0:
                        lam[k] += 1
                        heapq.heappush(heap, (-lam[k], k))
        for k in sp_idx[sp_ptr[i]:sp_ptr[i + 1]]:
            if state[k] == 0:
                lam[k] -= 1
                heapq.heappush(heap, (-lam[k], k))
    return np.asarray(state) == 1


def _direct_interpolation(A, S, is_c):
    """Direct interpolation: P_ij = -(alpha_i or beta_i) a_ij / a_ii over strong C neighbours."""
    n = A.shape[0]
    cidx = np.cumsum(is_c) - 1
    nc = int(is_c.sum())
    Ac = A.tocoo()
    off = Ac.row != Ac.col
    r, c, v = Ac.row[off], Ac.col[off], Ac.data[off]
    diag = A.diagonal()
    Sset = set(zip(*S.nonzero())) if S.nnz < 2_000_000 else None
    if Sset is not None:
        strong = np.fromiter(((ri, ci) in Sset for ri, ci in zip(r.tolist(), c.tolist())), bool, len(r))
    else:  # large matrices: strength pattern via a sorted-key lookup
        key = r.astype(np.int64) * n + c
        Sc = S.tocoo()
        skey = np.sort(Sc.row.astype(np.int64) * n + Sc.col)
        pos = np.searchsorted(skey, key)
        strong = (pos < len(skey)) & (skey[np.minimum(pos, len(skey) - 1)] == key)
    interp = strong & is_c[c] & ~is_c[r]
    neg = v < 0
    sum_neg = np.bincount(r, weights=np.where(neg, v, 0.0), minlength=n)
    sum_pos = np.bincount(r, weights=np.where(~neg, v, 0.0), minlength=n)
    csum_neg = np.bincount(r[interp], weights=np.where(neg[interp], v[interp], 0.0), minlength=n)
    csum_pos = np.bincount(r[interp], weights=np.where(~neg[interp], v[interp], 0.0), minlength=n)
    alpha = np.where(csum_neg != 0, sum_neg / np.where(csum_neg != 0, csum_neg, 1.0), 0.0)
    # positive off-diagonals with no positive C partner are lumped into the diagonal
    beta = np.where(csum_pos != 0, sum_pos / np.where(csum_pos != 0, csum_pos, 1.0), 0.0)
    dmod = diag + np.where(csum_pos == 0, sum_pos, 0.0)
    ri, ci, vi = r[interp], c[interp], v[interp]
    w = -np.where(vi < 0, alpha[ri], beta[ri]) * vi / dmod[ri]
    crow = np.nonzero(is_c)[0]
    rows = np.concatenate([crow, ri])
    cols = np.concatenate([cidx[crow], cidx[ci]])
    vals = np.concatenate([np.ones(nc), w])
    return _csr(sp.csr_matrix((vals, (rows, cols)), shape=(n, nc)))


def ruge_stuben_solver(A, max_levels=10, max_coarse=10, theta=0.25, **_ignored):
    """Build a classical (Ruge-Stueben) hierarchy with the defaults in the module docstring."""
    A = _csr(A).astype(np.float64)
    levels = [HostLevel(A)]
    while len(levels) < max_levels and levels[-1].A.shape[0] > max_coarse:
        A = levels[-1].A
        S = _classical_strength(A, theta)
        is_c = _rs_first_pass(S)
        nc = int(is_c.sum())
        if nc == 0 or nc >= A.shape[0]:
            break
        P = _direct_interpolation(A, S, is_c)
        R = _csr(P.T)
        levels[-1].P = P
        levels[-1].R = R
        levels.append(HostLevel(_csr(R @ A @ P)))
    return HostHierarchy(levels, kind="ruge_stuben")


# ---------------------------------------------------------------- AIR (nonsymmetric)

def _one_point_interpolation(A, S, is_c):
    """Each C point injects itself; each F point takes the value of its strongest C
    neighbour (largest |a_ij| among strong C connections), weight 1; F points without one
    get a zero row."""
    n = A.shape[0]
    cidx = np.cumsum(is_c) - 1
    Sc = S.tocoo()
    A_abs = abs(A).tocsr()
    vals = np.asarray(A_abs[Sc.row, Sc.col]).ravel()
    keep = is_c[Sc.col] & ~is_c[Sc.row]
    r, c, v = Sc.row[keep], Sc.col[keep], vals[keep]
    best = np.full(n, -1)
    bestv = np.full(n, -np.inf)
    order = np.lexsort((c, -v))  # strongest first, ties by column
    for ri, ci, vi in zip(r[order], c[order], v[order]):
        if best[ri] < 0:
            best[ri] = ci
            bestv[ri] = vi
    crow = np.nonzero(is_c)[0]
    frow = np.nonzero((~is_c) & (best >= 0))[0]
    rows = np.concatenate([crow, frow])
    cols = np.concatenate([cidx[crow], cidx[best[frow]]])
    return _csr(sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, int(is_c.sum()))))


def _air_restriction(A, S, is_c):
    """Distance-1 approximate ideal restriction.  The ideal restriction is
    R = [-A_cf A_ff^-1, I]; row i of R (a C point) is approximated on the F points N_i it
    strongly depends on by solving the local system z^T A[N_i, N_i] = -A[i, N_i], and
    carries 1 at i itself."""
    n = A.shape[0]
    cidx = np.cumsum(is_c) - 1
    A = _csr(A)
    S = _csr(S)
    rows, cols, vals = [], [], []
    for i in np.nonzero(is_c)[0]:
        nb = S.indices[S.indptr[i]:S.indptr[i + 1]]
        Ni = nb[~is_c[nb]]
        rows.append(cidx[i]); cols.append(i); vals.append(1.0)
        if len(Ni) == 0:
            continue
        Aff = A[Ni][:, Ni].toarray()
        aif = A[i, Ni].toarray().ravel()
        try:
            z = np.linalg.solve(Aff.T, -aif)
        except np.linalg.LinAlgError:
            z = np.linalg.lstsq(Aff.T, -aif, rcond=None)[0]
        rows.extend([cidx[i]] * len(Ni)); cols.extend(Ni.tolist()); vals.extend(z.tolist())
    return _csr(sp.csr_matrix((vals, (rows, cols)), shape=(int(is_c.sum()), n)))


def air_solver(A, max_levels=10, max_coarse=20, theta=0.3, **_ignored):
    """Approximate-ideal-restriction AMG for nonsymmetric (advection-dominated) problems
    (Manteuffel, Ruge, Southworth, SISC 2018): classical strength (theta = 0.3 on |a_ij|),
    first-pass Ruge-Stueben C/F splitting, one-point interpolation, distance-1 AIR
    restriction, Galerkin coarse operators R A P; R is not P^T."""
    A = _csr(A).astype(np.float64)
    levels = [HostLevel(A)]
    while len(levels) < max_levels and levels[-1].A.shape[0] > max_coarse:
        A = levels[-1].A
        S = _classical_strength(A, theta)
        is_c = _rs_first_pass(S)
        nc = int(is_c.sum())
        if nc == 0 or nc >= A.shape[0]:
            break
        P = _one_point_interpolation(A, S, is_c)
        R = _air_restriction(A, S, is_c)
        levels[-1].P = P
        levels[-1].R = R
        levels.append(HostLevel(_csr(R @ A @ P)))
    return HostHierarchy(levels, kind="air")


# ---------------------------------------------------------------- serialisation

def save_hierarchy(path, hierarchy):
    """Write every level's CSR arrays to one ``.npz`` (replayable on any machine)."""
    out = {"n_levels": np.array(len(hierarchy.levels)), "kind": np.array(getattr(hierarchy, "kind", ""))}
    for i, lvl in enumerate(hierarchy.levels):
        for name in ("A", "P", "R"):
            M = getattr(lvl, name, None)
            if M is None:
                continue
            M = _csr(M)
            out[f"{name}{i}_data"] = M.data
            out[f"{name}{i}_indices"] = M.indices.astype(np.int32)
            out[f"{name}{i}_indptr"] = M.indptr.astype(np.int64)
            out[f"{name}{i}_shape"] = np.array(M.shape)
    np.savez_compressed(path, **out)


def load_hierarchy(path):
    """Inverse of :func:`save_hierarchy`."""
    z = np.load(path, allow_pickle=False)
    levels = []
    for i in range(int(z["n_levels"])):
        mats = {}
        for name in ("A", "P", "R"):
            if f"{name}{i}_data" in z:
                mats[name] = sp.csr_matrix((z[f"{name}{i}_data"], z[f"{name}{i}_indices"], z[f"{name}{i}_indptr"]),
                                           shape=tuple(z[f"{name}{i}_shape"]))
        levels.append(HostLevel(mats["A"], mats.get("P"), mats.get("R")))
    return HostHierarchy(levels, kind=str(z["kind"]))
