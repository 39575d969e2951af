"""Smoother configuration (the interface of amjax/relaxation/smoothing.py).

A user writes a smoother as a name (``'jacobi'``), a ``(name, options)`` pair, ``None``
(no smoothing), or a list of those (one per level, the last repeated downwards).  This
module turns that into one resolved :class:`SmootherSpec` per level and, from it, the
level's callable.  The callable carries ``_amg_spec = (kind, iterations, omega)``, the
resolved numbers the native cycle reads; calling it runs the fused CUDA Jacobi sweep.

Kept identical to the reference because callers and its tests depend on them: the
exception types and messages (``ValueError`` for unknown or non-string names and bad
specs, smoothing.py:43-56,130-158; ``NotImplementedError`` for the names listed as not
implemented, smoothing.py:120-127), the ``symmetric_smoothing`` rule (same name, same
sweep count, name 'jacobi' or None; smoothing.py:212-228), ``withrho`` dividing omega by
the estimated spectral radius of D^-1 A once per level, and the per-level
``_presmoother_spec`` / ``_postsmoother_spec`` records with omega already resolved.
"""

from __future__ import annotations

from dataclasses import dataclass, field

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


@dataclass(frozen=True)
class SmootherSpec:
    """One level's smoother as the user wrote it: ``name`` (a string or None, unchanged)
    and its keyword options."""

    name: object
    options: dict = field(default_factory=dict)

    @staticmethod
    def of(item) -> "SmootherSpec":
        if isinstance(item, tuple):
            return SmootherSpec(item[0], item[1])
        return SmootherSpec(item, {})

    @property
    def sweeps(self):
        return self.options.get("iterations", DEFAULT_NITER)


def specs_per_level(spec, n_levels: int) -> list:
    """The smoother of each of ``n_levels`` levels: a single spec applies to all of them,
    a list gives level i its i-th entry and the last entry to every level beyond it."""
    if isinstance(spec, list):
        items = spec
    elif spec is None or isinstance(spec, (str, tuple)):
        items = [spec]
    else:
        raise ValueError(f"Unrecognized smoother specification: {spec!r}")
    if not items:
        raise ValueError("Empty smoother specification.")
    return [SmootherSpec.of(items[min(i, len(items) - 1)]) for i in range(n_levels)]


def setup_jacobi(lvl, iterations=DEFAULT_NITER, omega=1.0, withrho=False):
    """Damped Jacobi on ``lvl`` (smoothing.py:85-99).  ``withrho`` scales omega by
    1/rho(D^-1 A), the power-iteration estimate, computed once and kept on the level."""
    if withrho:
        rho = getattr(lvl, "_spectral_radius", None)
        if rho is None:
            rho = relaxation.approximate_spectral_radius(lvl.A, lvl.Dinv)
            lvl._spectral_radius = rho
        omega = omega / rho
    dinv = lvl.Dinv
    sweeps, w = int(iterations), float(omega)

    def jacobi_smoother(A, x, b):
        return relaxation.jacobi(A, x, b, dinv, iterations=sweeps, omega=w)

    jacobi_smoother.__name__ = "jacobi"
    jacobi_smoother._omega = omega
    jacobi_smoother._amg_spec = ("jacobi", sweeps, w)
    return jacobi_smoother


def setup_none(lvl, **kwargs):
    """The identity smoother (smoothing.py:102-117): returns x unchanged."""
    del lvl, kwargs

    def identity_smoother(A, x, b):
        return x

    identity_smoother.__name__ = "none"
    identity_smoother._amg_spec = ("none", 0, 1.0)
    return identity_smoother


_FACTORIES = {"jacobi": setup_jacobi, "none": setup_none}


def _factory(name):
    """The set-up function for ``name`` (None means 'none'), with the reference's errors."""
    key = "none" if name is None else name
    if not isinstance(key, str):
        raise ValueError(f"Smoother name must be a string or None, got {key!r}")
    if key in _NOT_IMPLEMENTED_SMOOTHERS:
        raise NotImplementedError(
            f"'{key}' smoother is not yet implemented in AMJax. Available: {sorted(_FACTORIES)}")
    try:
        return _FACTORIES[key]
    except KeyError:
        raise ValueError(f"Unknown smoother {key!r}. Available: {sorted(_FACTORIES)}") from None


def _resolved_options(spec: SmootherSpec, built) -> dict:
    """The options with a withrho-scaled omega written in (so a rebuild needs no rho)."""
    opts = dict(spec.options)
    if opts.get("withrho", False):
        opts.update(omega=built._omega, withrho=False)
    return opts


def _build(lvl, spec: SmootherSpec):
    fn = _factory(spec.name)(lvl, **spec.options)
    return fn, (spec.name, _resolved_options(spec, fn))


def _is_symmetric_pair(pre: SmootherSpec, post: SmootherSpec) -> bool:
    return pre.name == post.name and pre.sweeps == post.sweeps and pre.name in SYMMETRIC_RELAXATION


def change_smoothers(ml, presmoother, postsmoother):
    """Give every level but the coarsest its pre- and post-smoother (smoothing.py:161-228)
    and set ``ml.symmetric_smoothing``."""
    n = len(ml.levels) - 1
    if n <= 0:
        return
    pres = specs_per_level(presmoother, n)
    posts = specs_per_level(postsmoother, n)
    symmetric = True
    for lvl, pre, post in zip(ml.levels[:n], pres, posts):
        lvl.presmoother, lvl._presmoother_spec = _build(lvl, pre)
        lvl.postsmoother, lvl._postsmoother_spec = _build(lvl, post)
        symmetric = symmetric and _is_symmetric_pair(pre, post)
    ml.symmetric_smoothing = symmetric
    if hasattr(ml, "_invalidate"):
        ml._invalidate()


def rebuild_smoother(lvl):
    """Re-create a level's smoothers from its recorded specs (smoothing.py:231-254)."""
    recorded = []
    for attr, label in (("_presmoother_spec", "_presmoother_spec"), ("_postsmoother_spec", "_postsmoother_spec")):
        rec = getattr(lvl, attr, None)
        if rec is None:
            raise AttributeError(f"Missing {label} on level.")
        recorded.append(rec)
    (pre_name, pre_opts), (post_name, post_opts) = recorded
    lvl.presmoother = _factory(pre_name)(lvl, **pre_opts)
    lvl.postsmoother = _factory(post_name)(lvl, **post_opts)
