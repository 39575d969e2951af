"""Host-side API behaviour that needs no GPU: smoother spec parsing and its error rules
(amjax/relaxation/smoothing.py), coarse-solver error rules (amjax/multilevel.py:448-498),
complexities and repr formulas, hierarchy set-up and serialisation, the byte model."""

import numpy as np
import pytest
import scipy.sparse as sp

from amjax_b200 import amg_setup, bytemodel, gallery
from amjax_b200.multilevel import MultilevelSolver, _NOT_IMPLEMENTED_SOLVERS, coarse_grid_solver
from amjax_b200.relaxation import smoothing
from amjax_b200.relaxation.relaxation import approximate_spectral_radius, inverse_diagonal


class _FakeA:
    def __init__(self, n, nnz):
        self.shape = (n, n)
        self.nnz = nnz


class _Lvl:
    def __init__(self, A):
        self.A = A
        self.Dinv = inverse_diagonal(A)


class _FakeML:
    def __init__(self, levels):
        self.levels = levels
        self.symmetric_smoothing = False


def _fake_ml(n=20):
    host = amg_setup.ruge_stuben_solver(gallery.poisson((n,)))
    return _FakeML([_Lvl(l.A) for l in host.levels])


def test_cycle_complexity_known_answers():
    """tests/test_multilevel.py:110-153."""
    levels = []
    for n, nnz in [(10, 100), (5, 25), (3, 9), (2, 4)]:
        lvl = MultilevelSolver.Level()
        lvl.A = _FakeA(n, nnz)
        lvl.P = object()
        lvl.R = object()
        levels.append(lvl)
    for L, exp in [(1, (1.0, 1.0, 1.0)), (2, (2.25, 2.25, 2.25)), (3, (2.59, 3.18, 3.18)), (4, (2.72, 3.88, 3.66))]:
        mg = MultilevelSolver(levels[:L], None)
        np.testing.assert_allclose([mg.cycle_complexity(c) for c in "VWF"], exp)
        assert mg.operator_complexity() == sum(x for x in [100, 25, 9, 4][:L]) / 100
    with pytest.raises(NotImplementedError):
        MultilevelSolver(levels, None).cycle_complexity("AMLI")


@pytest.mark.parametrize("name", sorted(smoothing._NOT_IMPLEMENTED_SMOOTHERS))
def test_not_implemented_smoothers_raise(name):
    with pytest.raises(NotImplementedError):
        smoothing.change_smoothers(_fake_ml(), (name, {}), "jacobi")


def test_unknown_and_bad_smoother_specs():
    ml = _fake_ml()
    with pytest.raises(ValueError):
        smoothing.change_smoothers(ml, "bogus", None)
    with pytest.raises(ValueError):
        smoothing.change_smoothers(ml, (3, {}), None)
    with pytest.raises(ValueError):
        smoothing.change_smoothers(ml, 5, None)
    with pytest.raises(ValueError):
        smoothing.change_smoothers(ml, [], None)


def test_symmetric_smoothing_flags():
    """tests/relaxation/test_smoothing.py:40-63."""
    for method in [("jacobi", {"iterations": 1, "withrho": True}), ("jacobi", {"iterations": 2, "withrho": True}), None]:
        ml = _fake_ml()
        smoothing.change_smoothers(ml, method, method)
        assert ml.symmetric_smoothing
    for pre, post in [(("jacobi", {"iterations": 2}), ("jacobi", {"iterations": 1})), ("jacobi", None), (None, "jacobi")]:
        ml = _fake_ml()
        smoothing.change_smoothers(ml, pre, post)
        assert not ml.symmetric_smoothing


def test_withrho_bakes_omega():
    ml = _fake_ml()
    smoothing.change_smoothers(ml, ("jacobi", {"omega": 1.0, "withrho": True}), "jacobi")
    lvl = ml.levels[0]
    rho = approximate_spectral_radius(lvl.A, lvl.Dinv)
    assert lvl.presmoother._amg_spec == ("jacobi", 1, 1.0 / rho)
    assert lvl._presmoother_spec == ("jacobi", {"omega": 1.0 / rho, "withrho": False})
    assert lvl.postsmoother._amg_spec == ("jacobi", 1, 1.0)


def test_per_level_list_specs_and_rebuild():
    ml = _fake_ml()
    smoothing.change_smoothers(ml, [("jacobi", {"iterations": 3}), None], "jacobi")
    assert ml.levels[0].presmoother._amg_spec[:2] == ("jacobi", 3)
    assert all(l.presmoother.__name__ == "none" for l in ml.levels[1:-1])
    lvl = ml.levels[0]
    smoothing.rebuild_smoother(lvl)
    assert lvl.presmoother.__name__ == "jacobi" and lvl.postsmoother.__name__ == "jacobi"
    bare = MultilevelSolver.Level()
    with pytest.raises(AttributeError):
        smoothing.rebuild_smoother(bare)


@pytest.mark.parametrize("name", sorted(_NOT_IMPLEMENTED_SOLVERS))
def test_not_implemented_coarse_solvers_raise(name):
    with pytest.raises(NotImplementedError):
        coarse_grid_solver(name, MultilevelSolver.Level())


def test_unknown_coarse_solver_raises():
    with pytest.raises(ValueError):
        coarse_grid_solver("bad_solver", MultilevelSolver.Level())


def test_hierarchy_builders_and_npz_roundtrip(tmp_path):
    A = gallery.poisson((30, 30))
    for factory in (amg_setup.smoothed_aggregation_solver, amg_setup.ruge_stuben_solver,
                    amg_setup.rootnode_solver, amg_setup.pairwise_solver):
        h = factory(A)
        assert len(h.levels) > 1 and h.levels[-1].A.shape[0] <= 10 + 60
        for i, lvl in enumerate(h.levels[:-1]):
            nc = h.levels[i + 1].A.shape[0]
            assert lvl.P.shape == (lvl.A.shape[0], nc) and lvl.R.shape == (nc, lvl.A.shape[0])
            assert abs(h.levels[i + 1].A - lvl.R @ lvl.A @ lvl.P).max() < 1e-12
        p = tmp_path / "h.npz"
        amg_setup.save_hierarchy(p, h)
        g = amg_setup.load_hierarchy(p)
        assert len(g.levels) == len(h.levels)
        for a, b in zip(g.levels, h.levels):
            assert (a.A != b.A).nnz == 0


def test_gallery_shapes():
    assert gallery.poisson((500, 500)).nnz == 1_248_000
    assert gallery.poisson((48, 48, 48)).nnz == 760_320
    A = gallery.anisotropic_diffusion_2d(10, 1e-2)
    assert abs(A - A.T).max() < 1e-14
    C = gallery.convection_diffusion_2d(10)
    assert abs(C - C.T).max() > 0
    V = gallery.variable_diffusion_2d(16)
    assert abs(V - V.T).max() < 1e-12 and V.shape == (256, 256)


def test_bytemodel_monotone():
    stats = [{"n": 100, "nnz_A": 500, "nnz_P": 200, "nnz_R": 200}, {"n": 20, "nnz_A": 100, "nnz_P": 40, "nnz_R": 40},
             {"n": 4, "nnz_A": 16}]
    v = bytemodel.cycle_bytes(stats, 1, 8, "V")
    w = bytemodel.cycle_bytes(stats, 1, 8, "W")
    assert 0 < v < w
    assert bytemodel.solve_bytes(stats, 2, 10) > bytemodel.solve_bytes(stats, 1, 10)


def test_air_hierarchy_restriction_is_not_p_transpose():
    from oracle import amg_oracle as O
    C = gallery.convection_diffusion_2d(24, peclet=10.0)
    h = amg_setup.air_solver(C)
    assert len(h.levels) > 2
    lvl = h.levels[0]
    assert (lvl.R - lvl.P.T).count_nonzero() > 0
    for i, l in enumerate(h.levels[:-1]):
        assert abs(h.levels[i + 1].A - l.R @ l.A @ l.P).max() < 1e-12
    W = ("jacobi", {"iterations": 1, "omega": 2 / 3})
    ml = O.Hierarchy.from_host(h, presmoother=W, postsmoother=W)
    b = np.random.default_rng(0).standard_normal(C.shape[0])
    x, it, rr = O.solve_loop(ml, b, tol=1e-10, maxiter=200)
    assert rr < 1e-10 and it < 60


def test_spectral_radius_on_device_needs_a_cuda_matrix():
    import scipy.sparse as sp_
    A = sp_.diags([2.0, 2.0, 2.0]).tocsr()
    with pytest.raises(ValueError):
        approximate_spectral_radius(A, np.full(3, 0.5), on_device=True)


def test_rootnode_prolongation_keeps_its_constraints():
    """Root-node AMG (Manteuffel, Olson, Schroder & Southworth 2017): P injects at the root
    nodes, reproduces the candidate (P B_c = B on aggregated rows), and the energy
    minimisation lowers trace(P^T A P) below the tentative prolongator's."""
    import scipy.sparse as sp
    A = gallery.poisson((24, 24))
    S = amg_setup._symmetric_strength(amg_setup._csr(A))
    agg, nagg, roots = amg_setup._standard_aggregation(S, return_roots=True)
    B = np.ones((A.shape[0], 1))
    T, Bc = amg_setup._rootnode_tentative(agg, nagg, roots, B)
    P = amg_setup._energy_prolongation(amg_setup._csr(A), T, Bc, roots, np.nonzero(agg >= 0)[0])
    np.testing.assert_allclose(P[roots].toarray(), np.eye(nagg), atol=1e-14)
    np.testing.assert_allclose(P @ Bc[:, 0], B[:, 0], atol=1e-12)
    energy = lambda M: float((M.T @ (A @ M)).diagonal().sum())
    assert energy(P) < 0.9 * energy(T)
    assert np.all(np.isin(agg[roots], np.arange(nagg))) and len(set(roots.tolist())) == nagg


def test_pairwise_aggregates_hold_at_most_four_nodes():
    """Double pairwise aggregation (Notay 2010): unsmoothed piecewise-constant P, each
    aggregate (column) holds 1-4 fine nodes, each fine row at most one entry."""
    A = gallery.poisson((32, 32))
    h = amg_setup.pairwise_solver(A)
    P = h.levels[0].P
    assert set(np.unique(P.data).tolist()) == {1.0}
    assert np.diff(P.indptr).max() <= 1
    sizes = np.asarray(P.sum(axis=0)).ravel()
    assert sizes.min() >= 1 and sizes.max() <= 4
    assert P.shape[1] < A.shape[0] / 3


@pytest.mark.parametrize("factory", ["rootnode_solver", "pairwise_solver"])
def test_new_factories_converge_in_the_oracle(factory):
    """The hierarchies drive the FP64 oracle's V-cycle PCG and standalone solve to 1e-8."""
    from oracle import amg_oracle as O
    A = gallery.poisson((40, 40))
    h = getattr(amg_setup, factory)(A)
    W = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})
    oml = O.Hierarchy.from_host(h, presmoother=W, postsmoother=W)
    b = np.random.default_rng(0).standard_normal(A.shape[0])
    x, k = O.cg(A, b, tol=1e-8, maxiter=200, M=O.aspreconditioner(oml))
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b) and k < 60
    x, it, rr = O.solve_loop(oml, b, tol=1e-8, maxiter=400)
    assert rr < 1e-8
