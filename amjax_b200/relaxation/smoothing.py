"""Smoother set-up and configuration (amjax/relaxation/smoothing.py).

Host-side only: a smoother spec (``'jacobi'``, ``('jacobi', {...})``, a list, or
``None``) becomes one callable per level.  The callables carry their resolved
parameters (``_amg_spec = (kind, iterations, omega)``) which the native cycle reads;
calling one directly runs the fused Jacobi kernel.  Errors and flags follow the
reference: ``ValueError`` for unknown or non-string names (smoothing.py:144-156),
``NotImplementedError`` for the names the reference lists as not implemented
(smoothing.py:120-127), ``symmetric_smoothing`` as in smoothing.py:212-228.
"""

from __future__ import annotations

from . import relaxation

DEFAULT_NITER = 1
SYMMETRIC_RELAXATION = ["jacobi", None]

_NOT_IMPLEMENTED_SMOOTHERS = {
    "gauss_seidel", "sor", "block_jacobi", "block_gauss_seidel",
    "schwarz", "strength_based_schwarz", "richardson", "chebyshev",
    "jacobi_ne", "gauss_seidel_ne", "gauss_seidel_nr",
    "gauss_seidel_indexed", "cf_jacobi", "fc_jacobi",
    "cf_block_jacobi", "fc_block_jacobi", "gmres", "cg", "cgne", "cgnr",
    "bsr_gauss_seidel", "bsr_jacobi", "bsr_jacobi_indexed",
}


def _unpack_arg(v):
    """(name, kwargs) of a spec (smoothing.py:36-40)."""
    if isinstance(v, tuple):
        return v[0], v[1]
    return v, {}


def _as_list(v):
    """smoothing.py:43-49."""
    if isinstance(v, list):
        return v
    if isinstance(v, (str, tuple)) or v is None:
        return [v]
    raise ValueError(f"Unrecognized smoother specification: {v!r}")


def _expand_to_n(specs, n):
    """Repeat the last spec until there are n (smoothing.py:52-56)."""
    if not specs:
        raise ValueError("Empty smoother specification.")
    return (specs + [specs[-1]] * n)[:n]


def _bake_kwargs(kw, smoother):
    """Freeze a withrho-resolved omega into the kwargs (smoothing.py:59-82)."""
    if not kw.get("withrho", False):
        return dict(kw)
    return {**kw, "omega": smoother._omega, "withrho": False}


def setup_jacobi(lvl, iterations=DEFAULT_NITER, omega=1.0, withrho=False):
    """Damped Jacobi on this level (smoothing.py:85-99); withrho divides omega by the
    power-iteration estimate of rho(D^-1 A), computed once per level."""
    Dinv = lvl.Dinv
    if withrho:
        if not hasattr(lvl, "_spectral_radius"):
            lvl._spectral_radius = relaxation.approximate_spectral_radius(lvl.A, Dinv)
        omega = omega / lvl._spectral_radius

    def smoother(A, x, b):
        return relaxation.jacobi(A, x, b, Dinv, iterations=iterations, omega=omega)

    smoother.__name__ = "jacobi"
    smoother._omega = omega
    smoother._amg_spec = ("jacobi", int(iterations), float(omega))
    return smoother


def setup_none(lvl, **kwargs):
    """Identity smoother (smoothing.py:102-117)."""
    del lvl, kwargs

    def smoother(A, x, b):
        del A, b
        return x

    smoother.__name__ = "none"
    smoother._amg_spec = ("none", 0, 1.0)
    return smoother


def _setup_call(fn):
    """Registry lookup with the reference's error rules (smoothing.py:130-158)."""
    registry = {"jacobi": setup_jacobi, "none": setup_none}
    if fn is None:
        fn = "none"
    if not isinstance(fn, str):
        raise ValueError(f"Smoother name must be a string or None, got {fn!r}")
    if fn in _NOT_IMPLEMENTED_SMOOTHERS:
        raise NotImplementedError(
            f"'{fn}' smoother is not yet implemented in AMJax. Available: {sorted(registry)}")
    if fn not in registry:
        raise ValueError(f"Unknown smoother {fn!r}. Available: {sorted(registry)}")
    return registry[fn]


def change_smoothers(ml, presmoother, postsmoother):
    """Assign pre/post smoothers on every level but the coarsest
    (smoothing.py:161-228); sets ``ml.symmetric_smoothing``."""
    n = len(ml.levels[:-1])
    if n == 0:
        return
    pre_specs = _expand_to_n(_as_list(presmoother), n)
    post_specs = _expand_to_n(_as_list(postsmoother), n)
    ml.symmetric_smoothing = True
    for i in range(n):
        pre_fn, pre_kw = _unpack_arg(pre_specs[i])
        post_fn, post_kw = _unpack_arg(post_specs[i])
        lvl = ml.levels[i]
        lvl.presmoother = _setup_call(pre_fn)(lvl, **pre_kw)
        lvl.postsmoother = _setup_call(post_fn)(lvl, **post_kw)
        lvl._presmoother_spec = (pre_fn, _bake_kwargs(pre_kw, lvl.presmoother))
        lvl._postsmoother_spec = (post_fn, _bake_kwargs(post_kw, lvl.postsmoother))
        it1 = pre_kw.get("iterations", DEFAULT_NITER)
        it2 = post_kw.get("iterations", DEFAULT_NITER)
        if it1 != it2 or pre_fn != post_fn or pre_fn not in SYMMETRIC_RELAXATION:
            ml.symmetric_smoothing = False
    if hasattr(ml, "_invalidate"):
        ml._invalidate()


def rebuild_smoother(lvl):
    """Rebuild a level's smoothers from its stored specs (smoothing.py:231-254)."""
    if getattr(lvl, "_presmoother_spec", None) is None:
        raise AttributeError("Missing _presmoother_spec on level.")
    if getattr(lvl, "_postsmoother_spec", None) is None:
        raise AttributeError("Missing _postsmoother_spec on level.")
    fn1, kw1 = lvl._presmoother_spec
    fn2, kw2 = lvl._postsmoother_spec
    lvl.presmoother = _setup_call(fn1)(lvl, **kw1)
    lvl.postsmoother = _setup_call(fn2)(lvl, **kw2)
