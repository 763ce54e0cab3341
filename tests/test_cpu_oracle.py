"""The CPU FP64 restatement (oracle) against the reference's known answers
(tests/golden/known_answers.json, transcribed by tests/golden/make_golden.py)
and against dense least squares.  Runs without a GPU."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import as_solver_categories, dense_demeaned, generate_synthetic_data, normal_equation_residual

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))


def test_stable_argsort_cases(oracle):
    for case in GOLDEN["stable_argsort"]:
        key = np.array(case["key"], np.uint32)
        got = oracle.stable_argsort(key, case["n_levels"])
        np.testing.assert_array_equal(got, np.array(case["perm"], np.uint32))


@pytest.mark.parametrize("case", GOLDEN["design"], ids=lambda c: c["source"].split()[-1])
def test_design_locality_sort(oracle, case):
    cats = np.asfortranarray(np.array(case["columns"], np.uint32).T)
    s = oracle.OracleSolver(cats, cfg=oracle.precond_cfg("off"))
    perm = s.obs_perm()
    if case["obs_perm"] is None:
        assert perm is None
    else:
        np.testing.assert_array_equal(perm, case["obs_perm"])
    assert [s.term(t)[3] for t in range(len(case["columns"]))] == case["sorted"]


def test_slope_layout(oracle):
    c = GOLDEN["slope_layout"]
    eff = [oracle.Effect(np.array(c[t["levels"]], np.uint32), t["intercept"],
                         tuple(np.array(c[z]) for z in t["slopes"])) for t in c["terms"]]
    s = oracle.OracleSolver(eff, cfg=oracle.precond_cfg("off"))
    assert [s.term(t)[1] for t in range(3)] == c["offsets"]
    assert [s.term(t)[0] * s.term(t)[2] for t in range(3)] == c["n_dofs"]
    assert s.n_dofs == c["total_dofs"]


def test_level_means(oracle):
    c = GOLDEN["level_means"]
    cats = np.array(c["categories"], np.uint32).reshape(-1, 1)
    r = oracle.OracleSolver(cats).solve(np.array(c["y"]), tol=1e-12)
    assert r.converged
    np.testing.assert_allclose(r.x[:3], c["x"], atol=1e-9)


@pytest.mark.parametrize("case", GOLDEN["slopes"], ids=lambda c: c["source"].split()[-1])
def test_slopes_closed_form(oracle, case):
    lv = np.array(case["levels"], np.uint32)
    z = np.array(case["z"])
    y = np.array(case["y"])
    r = oracle.OracleSolver([oracle.Effect(lv, case["intercept"], (z,))]).solve(y)
    assert r.converged
    exp = np.array(case["x_expected"])
    assert np.all(np.abs(r.x - exp) <= 1e-6 * (1 + np.abs(exp)))


@pytest.mark.parametrize("case", GOLDEN["lsmr"], ids=lambda c: c["source"].split()[1])
def test_lsmr_fixtures(oracle, case):
    a = np.array(case["a"], np.float64)
    b = np.array(case["b"], np.float64)
    x, st = oracle.lsmr_dense(a, b, case["tol"], case["maxiter"], case.get("local_size", 0),
                              case.get("precond"))
    if "x" in case:
        assert np.linalg.norm(x - np.array(case["x"], float)) < case["x_tol"]
    if "x_rel" in case:
        ref = np.array(case["x_rel"])
        sc = np.max(np.abs(ref))
        assert np.linalg.norm((x - ref) / sc) / np.linalg.norm(ref / sc) < case["x_rel_tol"]
    if "normal_eq_max" in case and np.max(np.abs(b)) < 1e100:
        assert np.linalg.norm(a.T @ (b - a @ x)) < case["normal_eq_max"]
    if case.get("converged"):
        assert st.converged


def test_vec_norm(oracle):
    for v, n in GOLDEN["vec_norm"]["cases"]:
        assert oracle.vec_norm(np.array(v, float)) == n
    assert np.isfinite(oracle.vec_norm(np.array([1e300, 1e300])))
    assert np.isnan(oracle.vec_norm(np.array([np.nan])))
    assert np.isnan(oracle.vec_norm(np.array([0.0, np.nan])))


def test_coalesced_scatter_matches_naive(oracle):
    """scatter.rs:252-272: a sorted 70,000-row term with 1,000 levels and a
    slope, runs straddling chunk boundaries, against a naive scatter-add."""
    n, L = 70_000, 1_000
    levels = (np.arange(n) * L // n).astype(np.uint32)
    x = (np.arange(n) % 13).astype(float) - 6.0
    z = ((np.arange(n) * 7) % 11) / 11.0 - 0.5
    s = oracle.OracleSolver([oracle.Effect(levels, True, (z,))], cfg=oracle.precond_cfg("off"))
    zz = s.loading(0)  # whitened slope
    got = s.apply_adjoint(x)
    exp = np.concatenate([np.bincount(levels, weights=x, minlength=L),
                          np.bincount(levels, weights=zz * x, minlength=L)])
    np.testing.assert_allclose(got, exp, atol=1e-9)


@pytest.mark.parametrize("kind,exact", [("off", False), ("diagonal", False), ("additive", True),
                                        ("additive", False)])
def test_solution_matches_dense_lstsq(oracle, kind, exact):
    rng = np.random.default_rng(1)
    n = 4000
    cats = [rng.integers(0, 50, n), rng.integers(0, 30, n), rng.integers(0, 7, n)]
    y = rng.standard_normal(n)
    w = rng.lognormal(0, 1, n)
    r = oracle.OracleSolver(as_solver_categories(cats), weights=w,
                            cfg=oracle.precond_cfg(kind, exact_local=exact)).solve(y, tol=1e-11, maxiter=5000)
    assert r.converged
    ref = dense_demeaned(cats, y, w)
    assert np.max(np.abs(r.demeaned - ref)) / np.linalg.norm(y) < 1e-8
    assert normal_equation_residual(cats, y, r.demeaned, w) < 1e-8


def test_noise_free_recovery(oracle):
    cats, _, y = generate_synthetic_data([50, 50], 10_000, seed=7)
    r = oracle.OracleSolver(as_solver_categories(cats)).solve(y)
    assert r.converged
    assert np.max(np.abs(r.demeaned)) < 1e-6 * np.linalg.norm(y)


def test_exact_local_solver_is_one_shot_for_two_factors(oracle):
    """With exact local solves a two-factor design has a single subdomain whose
    local solve is the exact pseudo-inverse, so LSMR converges in one step."""
    rng = np.random.default_rng(2)
    n = 3000
    cats = [rng.integers(0, 40, n), rng.integers(0, 15, n)]
    y = rng.standard_normal(n)
    s = oracle.OracleSolver(as_solver_categories(cats), cfg=oracle.precond_cfg("additive", exact_local=True))
    assert s.n_subdomains == 1
    assert s.solve(y, tol=1e-10).iterations <= 2


def test_input_validation(oracle):
    cats = np.zeros((5, 1), np.uint32)
    with pytest.raises(oracle.OracleError):
        oracle.OracleSolver(cats, weights=np.array([1.0, -1, 1, 1, 1]))
    s = oracle.OracleSolver(cats)
    with pytest.raises(oracle.OracleError):
        s.solve(np.array([1.0, np.nan, 0, 0, 0]))
    with pytest.raises(oracle.OracleError):
        oracle.OracleSolver(np.array([[np.iinfo(np.uint32).max]], np.uint32))


def test_threaded_timing_mode_matches_reference_order(oracle):
    """The restatement's timing mode (all host threads, used only by the
    bench's CPU baseline and reference arm) solves the same system: demeaned
    vectors agree with the single-thread reference order to rounding, and the
    one-thread mode stays bitwise identical run to run."""
    from within_b200 import workloads as W
    n = 200_000
    codes = W.akm_panel(n=n, n_workers=n // 10, n_firms=n // 100, seed=8)
    y = W.akm_response(n, seed=9)
    s = oracle.OracleSolver(codes)
    try:
        oracle.lib().or_set_threads(1)
        a = s.solve(y, tol=1e-10, maxiter=2000)
        b = s.solve(y, tol=1e-10, maxiter=2000)
        oracle.lib().or_set_threads(4)
        c = s.solve(y, tol=1e-10, maxiter=2000)
    finally:
        oracle.lib().or_set_threads(1)
    assert np.array_equal(a.demeaned, b.demeaned)
    assert c.converged
    assert np.max(np.abs(a.demeaned - c.demeaned)) / np.max(np.abs(y)) < 1e-8


@pytest.mark.parametrize("case", GOLDEN["slope_drops"], ids=lambda c: c["source"].split()[-1])
def test_slope_rank_drops(oracle, case):
    """Rank drops, exact zeros and closed forms of tests/slopes.rs:157-326 on
    the restatement (the GPU runs the same cases in test_gpu_slopes.py)."""
    from conftest import check_slope_drop_case
    lv = np.array(case["levels"], np.uint32)
    zs = tuple(np.array(z) for z in case["slopes"])
    w = None if case["weights"] is None else np.array(case["weights"])
    kinds = ["additive", "diagonal"] if case["also_diagonal"] else ["additive"]
    for kind in kinds:
        s = oracle.OracleSolver([oracle.Effect(lv, True, zs)], weights=w, cfg=oracle.precond_cfg(kind))
        for yv in case["y"]:
            y = np.array(yv)
            r = s.solve(y)
            assert r.converged
            check_slope_drop_case(case, r.x, r.demeaned, s.unidentified(), r.iterations, y)
