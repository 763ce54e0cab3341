"""The warp-range segmented reductions (within_tuning.warp_ranges = 1 for
C^T and the adjoint's combines, 2 for every tile plan; segsweep.cuh)
against the oracle and against the block-tile engine: every
column bucket (K = 1, 2, 4, 8), FP64 and mixed precision, designs with empty
levels (empty segments in the adjoint and Schwarz plans), a slope term, a
deep round-scheduled factor, and run-to-run bitwise reproducibility."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import as_solver_categories, demeaned_errors

pytestmark = pytest.mark.gpu


def rel_inf(a, b, y):
    """max|a - b| / ||y||_2 (the contract's scaling), after checking
    max|a - b| / max|y| <= 1e-6."""
    e = demeaned_errors(a, b, y)
    assert e["inf_over_inf"] <= 1e-6, e
    return e["inf_over_l2"]

WR = {"warp_ranges": 2}
WR_ALL = {"warp_ranges": 2, "thread_per_segment": 0}   # also C, prolongation and every round


def _panel(n=300_000, seed=31):
    from within_b200 import workloads as WL
    return WL.akm_panel(n=n, n_workers=n // 10, n_firms=n // 100, seed=seed)


@pytest.mark.parametrize("tuning", [{"warp_ranges": 1}, WR, WR_ALL, {"warp_ranges": 1, "staged_sweep": 0}])
def test_warp_ranges_match_oracle_panel(wb, oracle, tuning):
    codes = _panel()
    y = np.random.default_rng(32).standard_normal(codes.shape[0])
    r = wb.Solver(codes, tuning=tuning).solve(y, wb.LsmrOptions(tol=1e-10, maxiter=3000))
    o = oracle.OracleSolver(codes).solve(y, tol=1e-10, maxiter=3000)
    assert r.converged
    assert rel_inf(r.demeaned, o.demeaned, y) < 1e-7


def test_warp_ranges_empty_levels_and_slopes(wb, oracle):
    """Unused levels (every third worker id and a block of firm ids never
    occur) give empty segments; a slope term adds loaded positions."""
    rng = np.random.default_rng(33)
    n = 120_000
    worker = 3 * rng.integers(0, 6_000, n)
    firm = rng.integers(0, 900, n)
    firm[firm >= 600] += 200
    year = rng.integers(0, 9, n)
    x = rng.standard_normal(n)
    for tuning in (WR, WR_ALL):
        wk, fm, yr = worker.astype(np.uint32), firm.astype(np.uint32), year.astype(np.uint32)
        eff = [wb.Effect(wk, True), wb.Effect(fm, True, [x]), wb.Effect(yr, True)]
        y = rng.standard_normal(n)
        r = wb.Solver(eff, tuning=tuning).solve(y, wb.LsmrOptions(tol=1e-10, maxiter=3000))
        o = oracle.OracleSolver([oracle.Effect(wk, True), oracle.Effect(fm, True, (x,)),
                                 oracle.Effect(yr, True)]).solve(y, tol=1e-10, maxiter=3000)
        assert r.converged
        assert rel_inf(r.demeaned, o.demeaned, y) < 1e-7


@pytest.mark.parametrize("k", [2, 4, 8])
def test_warp_ranges_batched_match_tiles(wb, k):
    codes = _panel(n=200_000, seed=34)
    Y = np.asfortranarray(np.random.default_rng(35).standard_normal((codes.shape[0], k)))
    opts = wb.LsmrOptions(tol=1e-11, maxiter=3000)
    a = wb.Solver(codes, tuning={"warp_ranges": 0}).solve_batch(Y, opts)
    b = wb.Solver(codes, tuning=WR_ALL).solve_batch(Y, opts)
    for j in range(k):
        assert rel_inf(b.demeaned[:, j], a.demeaned[:, j], Y[:, j]) < 1e-8


def test_warp_ranges_mixed_precision(wb):
    codes = _panel(n=300_000, seed=36)
    rng = np.random.default_rng(37)
    w = rng.lognormal(0.0, 1.0, codes.shape[0])
    Y = np.asfortranarray(rng.standard_normal((codes.shape[0], 4)))
    ref = wb.Solver(codes, weights=w, tuning={"warp_ranges": 0}).solve_batch(Y, wb.LsmrOptions(tol=1e-12,
                                                                                               maxiter=5000))
    mx = wb.Solver(codes, weights=w, precision="mixed", tuning=WR).solve_batch(Y, wb.LsmrOptions(tol=1e-11,
                                                                                                 maxiter=5000))
    for j in range(4):
        assert mx.converged[j]
        d = np.max(np.abs(mx.demeaned[:, j] - ref.demeaned[:, j]))
        assert d / np.max(np.abs(Y[:, j])) < 1e-8


def test_warp_ranges_bitwise_reproducible(wb):
    codes = _panel(n=250_000, seed=38)
    y = np.random.default_rng(39).standard_normal(codes.shape[0])
    s = wb.Solver(codes, tuning=WR_ALL)
    opts = wb.LsmrOptions(tol=1e-9)
    a = s.solve(y, opts)
    b = s.solve(y, opts)
    c = wb.Solver(codes, tuning=WR_ALL).solve(y, opts)
    assert np.array_equal(a.demeaned, b.demeaned) and np.array_equal(a.x, b.x)
    assert np.array_equal(a.demeaned, c.demeaned)


def test_warp_ranges_deep_factor(wb, oracle):
    """A 3,000-level uniform design: its reduced system takes the small-graph
    rounds (a deep schedule with a fused tail) on warp ranges."""
    rng = np.random.default_rng(40)
    n = 150_000
    cats = as_solver_categories([rng.integers(0, 20_000, n), rng.integers(0, 3_000, n), rng.integers(0, 12, n)])
    y = rng.standard_normal(n)
    for tuning in (WR, WR_ALL, {"warp_ranges": 2, "fuse_rounds": 0}):
        r = wb.Solver(cats, tuning=tuning).solve(y, wb.LsmrOptions(tol=1e-10, maxiter=3000))
        o = oracle.OracleSolver(cats).solve(y, tol=1e-10, maxiter=3000)
        assert r.converged
        assert rel_inf(r.demeaned, o.demeaned, y) < 1e-7
