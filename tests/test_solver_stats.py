"""`duplicate`, `merge_stats!` and `solver_report` (src/ElasticitySplitNode.jl:
408-447) on the host side: no GPU involved."""
import pytest


def _stats(s, solves, iterations, max_it, unconv):
    s.stats.solves, s.stats.iterations = solves, iterations
    s.stats.max_iterations, s.stats.unconverged = max_it, unconv


def test_duplicate_keeps_options_and_resets_counters(eqd):
    s = eqd.CGSolver(None, rtol=1e-9, atol=1e-3, itmax=77, precond="jacobi", precision="fp64", chunk=5,
                     variant=3, split=False)
    _stats(s, 4, 100, 30, 1)
    d = eqd.duplicate(s)
    assert d is not s and d.fe is s.fe
    for k in ("rtol", "atol", "itmax", "precond", "precision", "chunk", "reliable_delta", "variant", "split", "fuse"):
        assert getattr(d, k) == getattr(s, k), k
    assert d.stats.solves == 0 and d.stats.iterations == 0 and d.stats.unconverged == 0


def test_merge_stats_folds_counters(eqd):
    a, b = eqd.CGSolver(None), eqd.CGSolver(None)
    _stats(a, 3, 90, 40, 0)
    _stats(b, 5, 100, 35, 2)
    out = eqd.merge_stats(a, b)
    assert out is a
    r = eqd.solver_report(a)
    assert r == dict(kind="cg", precond="none", solves=8, iterations=190, mean_iterations=190 / 8,
                     max_iterations=40, unconverged=2)
    assert eqd.solver_report(b)["solves"] == 5


def test_report_of_fresh_solver(eqd):
    r = eqd.solver_report(eqd.CGSolver(None, precond="jacobi"))
    assert r["solves"] == 0 and r["mean_iterations"] == 0.0 and r["precond"] == "jacobi"


def test_bad_options_raise(eqd):
    with pytest.raises(ValueError):
        eqd.CGSolver(None, precond="amg")
    with pytest.raises(ValueError):
        eqd.CGSolver(None, precision="fp16")
