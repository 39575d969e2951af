"""Shared fixtures: hierarchies and the oracle wrapper (the oracle is the checker)."""

import functools

import numpy as np

from amjax_b200 import amg_setup, gallery
from oracle import amg_oracle as O


@functools.lru_cache(maxsize=None)
def host_hierarchy(kind: str, n: int, dim: int = 2):
    A = gallery.poisson((n,) * dim)
    if kind == "sa":
        return amg_setup.smoothed_aggregation_solver(A)
    if kind == "rs":
        return amg_setup.ruge_stuben_solver(A)
    if kind == "rootnode":
        return amg_setup.rootnode_solver(A)
    if kind == "pairwise":
        return amg_setup.pairwise_solver(A)
    raise ValueError(kind)


def oracle_ml(host, pre=("jacobi", {"iterations": 1, "omega": 2.0 / 3.0}), post=None, coarse="pinv",
              coarse_kwargs=None, dtype=np.float64):
    post = pre if post is None else post
    return O.Hierarchy.from_host(host, presmoother=pre, postsmoother=post, coarse_solver=coarse,
                                 coarse_solver_kwargs=coarse_kwargs, dtype=dtype)


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
