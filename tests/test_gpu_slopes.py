"""Varying slopes on the GPU: back-transformed coefficients ``x`` in the
user's parametrisation, unidentified directions and their exact zeros.

- The reference's slope tests (tests/slopes.rs:96-326, transcribed into
  tests/golden/known_answers.json) run through the GPU solver: per-level
  closed forms, rank drops reported in ascending (level, column) order with
  x exactly 0.0 at the dropped slots (solver/reparam.rs:78-194), zero-weight
  rows masked out of identification, a batch sharing the unidentified list,
  three collinear slopes.
- A 2,000,000-row, 50,000-firm intercept + slope term (the firm term of the
  differentiable-demeaning panel, weights lognormal(0, 0.5)) against the
  per-level weighted OLS closed form, with planted rank drops: an empty
  level, a level whose covariate is constant, and the levels that hold a
  single observation by chance.
- The same firm term beside a 30-level year term: the slope coefficients
  (identified, unlike the intercepts, which share one constant per
  connected component) against the oracle.

Tolerances: |x - expected| <= 1e-6 (1 + |expected|), the reference's
assert_close (tests/slopes.rs:7-14); dropped slots exactly 0.0.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import check_slope_drop_case, demeaned_errors

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))


def drops(res):
    return [(d.term, d.level, d.column) for d in res.unidentified]


@pytest.mark.parametrize("case", GOLDEN["slopes"], ids=lambda c: c["source"].split()[-1])
def test_slopes_closed_form_on_gpu(wb, case):
    lv = np.array(case["levels"], np.uint32)
    z = np.array(case["z"])
    y = np.array(case["y"])
    r = wb.Solver([wb.Effect(lv, case["intercept"], [z])]).solve(y)
    assert r.converged and not r.unidentified
    exp = np.array(case["x_expected"])
    assert np.all(np.abs(r.x - exp) <= 1e-6 * (1 + np.abs(exp)))
    nl = int(lv.max()) + 1
    fitted = (r.x[lv] + r.x[nl + lv] * z) if case["intercept"] else r.x[lv] * z
    assert np.all(np.abs((y - r.demeaned) - fitted) <= 1e-6 * (1 + np.abs(fitted)))


@pytest.mark.parametrize("case", GOLDEN["slope_drops"], ids=lambda c: c["source"].split()[-1])
def test_slope_rank_drops_on_gpu(wb, case):
    lv = np.array(case["levels"], np.uint32)
    zs = [np.array(z) for z in case["slopes"]]
    w = None if case["weights"] is None else np.array(case["weights"])
    pcs = [None, wb.PreconditionerConfig.Diagonal] if case["also_diagonal"] else [None]
    xs = []
    for pc in pcs:
        s = wb.Solver([wb.Effect(lv, True, zs)], weights=w, preconditioner=pc)
        for yv in case["y"]:
            y = np.array(yv)
            r = s.solve(y)
            assert r.converged
            check_slope_drop_case(case, r.x, r.demeaned, drops(r), r.iterations, y)
            xs.append(r.x)
        if len(case["y"]) > 1:   # batch: shared unidentified list, each column its own back-transform
            Y = np.asfortranarray(np.column_stack([np.array(v) for v in case["y"]]))
            b = s.solve_batch(Y)
            assert [(d.term, d.level, d.column) for d in b.unidentified] == [tuple(t) for t in case["drops"]]
            for j, yv in enumerate(case["y"]):
                single = s.solve(np.array(yv))
                assert np.all(np.abs(b.x[:, j] - single.x) <= 1e-9 * (1 + np.abs(single.x)))
                for slot in case["zero_slots"]:
                    assert b.x[slot, j] == 0.0
    if len(pcs) == 2:   # the explicit diagonal preconditioner agrees with the default path
        assert np.all(np.abs(xs[1] - xs[0]) <= 1e-6 * (1 + np.abs(xs[0])))


def firm_slope_panel():
    """The firm term of the 2M-row varying-slopes panel with planted drops:
    firm 0's rows move to firm 1 (firm 0 empty: intercept and slope drop),
    firm 2's covariate is set constant (its slope drops)."""
    from within_b200 import workloads as WL
    firm, year, x, z, w, v = WL.slopes_panel()
    firm = firm.copy()
    x = x.copy()
    firm[firm == 0] = 1
    x[firm == 2] = 0.7
    return firm, year, x, z, w


def closed_form(firm, x, y, w, n_levels):
    """Per-level weighted OLS of y on [1, x] (tests/slopes.rs:19-45) with the
    drop rule of solver/reparam.rs:78-194 for one slope: the intercept drops
    when a level has no positive-weight row, the slope when its positive-weight
    rows hold fewer than two distinct covariate values (centred Gram exactly 0)."""
    pos = w > 0
    f, xx, yy, ww = firm[pos], x[pos], y[pos], w[pos]
    sw = np.bincount(f, ww, n_levels)
    safe = np.where(sw > 0, sw, 1.0)
    mx = np.bincount(f, ww * xx, n_levels) / safe
    my = np.bincount(f, ww * yy, n_levels) / safe
    dx, dy = xx - mx[f], yy - my[f]   # centred sums: no cancellation on close covariates
    cxx = np.bincount(f, ww * dx * dx, n_levels)
    cxy = np.bincount(f, ww * dx * dy, n_levels)
    xmin = np.full(n_levels, np.inf)
    xmax = np.full(n_levels, -np.inf)
    np.minimum.at(xmin, f, xx)
    np.maximum.at(xmax, f, xx)
    slope_ok = (sw > 0) & (xmax > xmin)
    b = np.where(slope_ok, cxy / np.where(slope_ok, cxx, 1.0), 0.0)
    a = np.where(sw > 0, my - b * mx, 0.0)
    expected_drops = []
    for lvl in np.flatnonzero((sw == 0) | ~slope_ok):
        if sw[lvl] == 0:
            expected_drops.append((0, int(lvl), 0))
        expected_drops.append((0, int(lvl), 1))
    return a, b, slope_ok, sw > 0, expected_drops


def test_firm_slope_term_2m_rows_closed_form(wb):
    firm, _, x, _, w = firm_slope_panel()
    y = np.random.default_rng(51).standard_normal(firm.size) + 0.3 * x
    nl = int(firm.max()) + 1
    a, b, slope_ok, icpt_ok, expected_drops = closed_form(firm, x, y, w, nl)
    assert (0, 0, 0) in expected_drops and (0, 2, 1) in expected_drops
    # One term has no factor pair, so the default preconditioner falls back to
    # none (operator/schwarz.rs:249-252) and A'A = diag(sum of w per level, 1)
    # is as ill-conditioned as the firm sizes; the diagonal preconditioner
    # makes it the identity, so the solve is exact and x is judged alone.
    s = wb.Solver([wb.Effect(firm, True, [x])], weights=w, preconditioner=wb.PreconditionerConfig.Diagonal)
    r = s.solve(y)
    assert r.converged
    assert drops(r) == expected_drops
    zero = np.concatenate([np.flatnonzero(~icpt_ok), nl + np.flatnonzero(~slope_ok)])
    assert np.all(r.x[zero] == 0.0)
    ok = np.flatnonzero(icpt_ok)
    assert np.all(np.abs(r.x[ok] - a[ok]) <= 1e-6 * (1 + np.abs(a[ok])))
    ok = np.flatnonzero(slope_ok)
    assert np.all(np.abs(r.x[nl + ok] - b[ok]) <= 1e-6 * (1 + np.abs(b[ok])))
    fitted = r.x[firm] + r.x[nl + firm] * x
    assert np.max(np.abs((y - r.demeaned) - fitted)) <= 1e-6 * (1 + np.max(np.abs(fitted)))


def test_firm_slope_and_year_2m_rows_slopes_match_oracle(wb, oracle):
    """Two terms (firm intercept + slope, year intercept), weighted: the firm
    slopes are unique, so they are compared with the oracle's directly; the
    demeaned vectors in both scalings."""
    firm, year, x, z, w = firm_slope_panel()
    nl = int(firm.max()) + 1
    opts = wb.LsmrOptions(tol=1e-10, maxiter=5000)
    s = wb.Solver([wb.Effect(firm, True, [x]), wb.Effect(year, True)], weights=w)
    r = s.solve(z, opts)
    oracle.lib().or_set_threads(os.cpu_count() or 1)
    try:
        o = oracle.OracleSolver([oracle.Effect(firm, True, (x,)), oracle.Effect(year, True)], weights=w)
        ro = o.solve(z, tol=1e-10, maxiter=5000)
        assert [tuple(t) for t in o.unidentified()] == drops(r)
    finally:
        oracle.lib().or_set_threads(1)
    assert r.converged and ro.converged
    _, _, slope_ok, _, _ = closed_form(firm, x, z, w, nl)
    sl = nl + np.flatnonzero(slope_ok)
    d = np.abs(r.x[sl] - ro.x[sl])
    assert np.max(d / (1 + np.abs(ro.x[sl]))) <= 1e-6
    dropped = nl + np.flatnonzero(~slope_ok)
    assert np.all(r.x[dropped] == 0.0)
    e = demeaned_errors(r.demeaned, ro.demeaned, z)
    assert e["inf_over_l2"] <= 1e-7 and e["inf_over_inf"] <= 1e-6, e
