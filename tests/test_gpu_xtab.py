"""The GPU cross-tabs of the additive-Schwarz set-up (within_tuning
gpu_cross_tab, xtab.cu) against the host accumulation: the serialised
preconditioner (every array of the host image) must be the same bytes, and
so must the solves, for unweighted and weighted designs, zero weights, a
slope term, unused levels and a design above the default size threshold."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(wb, design, weights=None):
    off = wb.Solver(design, weights=weights, tuning={"gpu_cross_tab": 0})
    on = wb.Solver(design, weights=weights, tuning={"gpu_cross_tab": 2})
    return off, on


def _same(wb, design, weights=None, y=None):
    off, on = _pair(wb, design, weights)
    assert off.preconditioner.to_bytes() == on.preconditioner.to_bytes()
    if y is not None:
        opts = wb.LsmrOptions(tol=1e-9)
        a, b = off.solve(y, opts), on.solve(y, opts)
        np.testing.assert_array_equal(a.demeaned, b.demeaned)
        np.testing.assert_array_equal(a.x, b.x)


def test_gpu_cross_tab_unweighted_three_terms(wb):
    rng = np.random.default_rng(51)
    n = 60_000
    cats = np.asfortranarray(np.column_stack([rng.integers(0, 6_000, n), rng.integers(0, 700, n),
                                              rng.integers(0, 9, n)]).astype(np.uint32))
    _same(wb, cats, y=rng.standard_normal(n))


def test_gpu_cross_tab_weighted_zero_weights_and_unused_levels(wb):
    rng = np.random.default_rng(52)
    n = 50_000
    w = rng.lognormal(0.0, 1.0, n)
    w[rng.random(n) < 0.15] = 0.0
    cats = np.asfortranarray(np.column_stack([2 * rng.integers(0, 4_000, n), rng.integers(0, 300, n),
                                              rng.integers(0, 7, n)]).astype(np.uint32))
    _same(wb, cats, weights=w, y=rng.standard_normal(n))


def test_gpu_cross_tab_slope_term(wb):
    rng = np.random.default_rng(53)
    n = 40_000
    f = rng.integers(0, 900, n).astype(np.uint32)
    g = rng.integers(0, 3_000, n).astype(np.uint32)
    yr = rng.integers(0, 11, n).astype(np.uint32)
    x = rng.standard_normal(n)
    w = rng.lognormal(0.0, 0.5, n)
    eff = [wb.Effect(g, True), wb.Effect(f, True, [x]), wb.Effect(yr, True)]
    _same(wb, eff, weights=w, y=rng.standard_normal(n))


def test_gpu_cross_tab_default_threshold_panel(wb):
    """A 400,000-row panel takes the GPU cross-tabs by default (at least 2^18
    observations) and gives the host image; its round-scheduled factor is
    built from them."""
    from within_b200 import workloads as WL
    codes = WL.akm_panel(n=400_000, n_workers=40_000, n_firms=4_000, seed=54)
    off = wb.Solver(codes, tuning={"gpu_cross_tab": 0})
    dflt = wb.Solver(codes)
    assert off.preconditioner.to_bytes() == dflt.preconditioner.to_bytes()
