"""Many independent designs (SolverSet / within_solvers_*): every design's
result equals its own Solver's bit for bit (the concurrent drive changes no
arithmetic), one design against the restatement, and error propagation."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_designs(count=7, seed=1):
    from within_b200 import workloads as W
    return W.many_designs(count=count, lo=3_000, hi=60_000, k=3, seed=seed)


def test_solver_set_matches_single_solvers(wb):
    cases = small_designs()
    rng = np.random.default_rng(0)
    weights = [None if i % 2 else rng.lognormal(0, 0.5, c.shape[0]) for i, (c, _) in enumerate(cases)]
    opts = wb.LsmrOptions(tol=1e-9, maxiter=5000)
    ss = wb.SolverSet([c for c, _ in cases], weights=weights, threads=4)
    assert len(ss) == len(cases)
    out = ss.solve_batch([Y for _, Y in cases], opts)
    for i, (codes, Y) in enumerate(cases):
        single = wb.Solver(codes, weights=weights[i]).solve_batch(Y, opts)
        x, dm, conv, its = out[i]
        assert all(conv)
        np.testing.assert_array_equal(dm, single.demeaned)
        np.testing.assert_array_equal(x, single.x)
        assert its == single.iterations


def test_solve_many_against_restatement(wb, oracle):
    cases = small_designs(count=3, seed=4)
    res = wb.solve_many([c for c, _ in cases], [Y for _, Y in cases], options=wb.LsmrOptions(tol=1e-10,
                                                                                          maxiter=5000))
    codes, Y = cases[2]
    o = oracle.OracleSolver(codes, cfg=oracle.precond_cfg("diagonal"))
    for c in range(Y.shape[1]):
        ref = o.solve(np.ascontiguousarray(Y[:, c]), tol=1e-11, maxiter=20000).demeaned
        assert np.max(np.abs(res[2][1][:, c] - ref)) / np.max(np.abs(Y[:, c])) < 1e-7


def test_solver_set_errors(wb):
    cases = small_designs(count=2)
    with pytest.raises(ValueError):
        wb.SolverSet([c for c, _ in cases], weights=[np.ones(5), None])
    ss = wb.SolverSet([c for c, _ in cases])
    with pytest.raises(ValueError):
        ss.solve_batch([cases[0][1]])
    bad = cases[1][1].copy()
    bad[3, 0] = np.nan
    with pytest.raises(ValueError):
        ss.solve_batch([cases[0][1], bad])


def test_solver_set_mixed_precision_matches_single_mixed_solvers(wb):
    """The FP32-with-FP64-refinement variant of the many-designs batch: every
    design equals its own mixed-precision Solver bit for bit, and lies within
    1e-7 (max|d| / max|y|) of the FP64 solve at tol 1e-11."""
    cases = small_designs(count=5, seed=2)
    opts = wb.LsmrOptions(tol=1e-10, maxiter=5000)
    ss = wb.SolverSet([c for c, _ in cases], threads=4, precision="mixed")
    out = ss.solve_batch([Y for _, Y in cases], opts)
    for i, (codes, Y) in enumerate(cases):
        single = wb.Solver(codes, precision="mixed").solve_batch(Y, opts)
        x, dm, conv, its = out[i]
        assert all(conv)
        np.testing.assert_array_equal(dm, single.demeaned)
        ref = wb.Solver(codes).solve_batch(Y, wb.LsmrOptions(tol=1e-11, maxiter=5000))
        for c in range(Y.shape[1]):
            assert np.max(np.abs(dm[:, c] - ref.demeaned[:, c])) <= 1e-7 * np.max(np.abs(Y[:, c]))
    ss.set_precision("fp64")
    out64 = ss.solve_batch([Y for _, Y in cases], opts)
    single64 = wb.Solver(cases[0][0]).solve_batch(cases[0][1], opts)
    np.testing.assert_array_equal(out64[0][1], single64.demeaned)
