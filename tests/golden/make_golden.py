"""Writes tests/golden/known_answers.json: the known-answer cases of the
reference's own tests for this path, with their expected values.

The reference (Rust + PyO3) cannot be built or imported in this environment,
so its test inputs and expected outputs are transcribed here; where the
reference test computes its expectation in closed form (per-level OLS,
stable sort, level means) the same closed form is evaluated with numpy.
Each case names the reference test it comes from.  Run:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def xorshift_keys():
    """crates/within/src/domain.rs:356-391 -- stable_argsort_branches_agree_with_a_stable_reference."""
    mask = (1 << 64) - 1
    state = 0x2545_F491_4F6C_DD1D
    cases = []
    for n_obs, n_levels, key_span in [(0, 0, 1), (0, 4, 4), (1, 1, 1), (997, 1, 1), (997, 16, 16),
                                      (997, 996, 996), (997, 997, 997), (997, 998, 998),
                                      (997, 50_000, 50_000), (4096, 4096, 8), (4096, 4096, 4096)]:
        key = []
        for _ in range(n_obs):
            state ^= (state << 13) & mask
            state ^= state >> 7
            state ^= (state << 17) & mask
            key.append(state % key_span)
        expected = sorted(range(n_obs), key=lambda i: key[i])  # Python's sort is stable
        cases.append({"n_levels": n_levels, "key": key, "perm": expected})
    return cases


def design_cases():
    """crates/within/src/domain.rs:394-519 (design build / locality sort tests)."""
    return [
        {"source": "domain.rs from_frame_sorts_owned_unsorted_dominant",
         "columns": [[2, 0, 1, 0], [0, 0, 1, 1]], "obs_perm": [1, 3, 2, 0], "sorted": [True, False],
         "internal": [[0, 0, 1, 2], [0, 1, 1, 0]]},
        {"source": "domain.rs rescan_marks_nested_factor_sorted_after_permutation",
         "columns": [[3, 0, 2, 1], [1, 0, 1, 0]], "obs_perm": [1, 3, 2, 0], "sorted": [True, True],
         "internal": [[0, 1, 2, 3], [0, 0, 1, 1]]},
        {"source": "domain.rs from_frame_keeps_sorted_input",
         "columns": [[0, 0, 1, 2], [1, 0, 1, 0]], "obs_perm": None, "sorted": [True, False],
         "internal": [[0, 0, 1, 2], [1, 0, 1, 0]]},
    ]


def slope_layout_case():
    """domain.rs new_lays_out_slope_terms_term_major: term offsets 0, 6, 9; n_dofs 11."""
    return {"f0": [0, 0, 1, 1], "f1": [0, 2, 1, 0], "z0": [1.0, 2.0, 3.0, 4.0],
            "z1": [5.0, 6.0, 7.0, 8.0],
            "terms": [{"levels": "f0", "intercept": True, "slopes": ["z0", "z1"]},
                      {"levels": "f1", "intercept": True, "slopes": []},
                      {"levels": "f0", "intercept": False, "slopes": ["z1"]}],
            "offsets": [0, 6, 9], "n_dofs": [6, 3, 2], "total_dofs": 11}


def per_level_ols(levels, z, y, n_levels):
    """tests/slopes.rs:19-45 -- per-level OLS of y on [1, z]."""
    a, b = [], []
    for lv in range(n_levels):
        m = levels == lv
        sw, sz, szz = m.sum(), z[m].sum(), (z[m] ** 2).sum()
        sy, szy = y[m].sum(), (z[m] * y[m]).sum()
        den = sw * szz - sz * sz
        bb = (sw * szy - sz * sy) / den
        a.append((sy - bb * sz) / sw)
        b.append(bb)
    return a, b


def slope_cases():
    synthetic_y = lambda n: [math.sin(i * 0.9 - 1.0) * 2.0 + 0.5 for i in range(n)]  # noqa: E731
    lv = np.array([2, 0, 1, 2, 0, 1, 2, 0, 1, 2, 0, 1])
    z = np.array([0.5, -1.2, 3.3, 1.5, 0.7, -2.1, 2.5, 1.9, 0.4, -0.5, -1.0, 1.1])
    y = np.array(synthetic_y(len(lv)))
    a, b = per_level_ols(lv, z, y, 3)
    lv2 = np.array([0, 0, 0, 1, 1, 1, 2, 2, 2])
    z2 = np.array([1.0, 2.0, -1.5, 0.5, 3.0, 1.0, -2.0, 0.7, 1.3])
    y2 = np.array(synthetic_y(len(lv2)))
    b2 = [float((z2[lv2 == l] * y2[lv2 == l]).sum() / (z2[lv2 == l] ** 2).sum()) for l in range(3)]
    return [
        {"source": "tests/slopes.rs single_slope_recovers_per_level_ols_and_fitted_values",
         "levels": lv.tolist(), "z": z.tolist(), "y": y.tolist(), "intercept": True,
         "x_expected": [float(v) for v in a + b]},
        {"source": "tests/slopes.rs slope_only_term_recovers_per_level_projection",
         "levels": lv2.tolist(), "z": z2.tolist(), "y": y2.tolist(), "intercept": False,
         "x_expected": b2},
    ]


def weighted_per_level_ols(levels, z, y, w, n_levels):
    """tests/slopes.rs:19-45 with weights: per-level weighted OLS of y on [1, z]."""
    a, b = [], []
    for lv in range(n_levels):
        m = levels == lv
        sw = w[m].sum()
        sz = (w[m] * z[m]).sum()
        szz = (w[m] * z[m] * z[m]).sum()
        sy = (w[m] * y[m]).sum()
        szy = (w[m] * z[m] * y[m]).sum()
        den = sw * szz - sz * sz
        bb = (sw * szy - sz * sy) / den if den != 0 else float("nan")
        a.append(float((sy - bb * sz) / sw) if sw != 0 else float("nan"))
        b.append(float(bb))
    return a, b


def slope_drop_cases():
    """tests/slopes.rs:157-326 -- rank drops with exact zeros, zero-weight
    masking, batch sharing and three collinear slopes.  Each case gives the
    reference's expected unidentified (term, level, column) triples, the x
    slots that must read exactly 0.0, and closed-form values for the
    identified slots ("checks": [slot, expected])."""
    synthetic_y = lambda n: np.array([math.sin(i * 0.9 - 1.0) * 2.0 + 0.5 for i in range(n)])  # noqa: E731
    cases = []
    # rank_drops_report_deterministically_with_exact_zeros: level 1 never
    # occurs, level 2's slope is constant
    lv = np.array([0, 0, 0, 2, 2, 2, 3, 3, 3])
    z = np.array([1.0, 2.0, -1.5, 2.5, 2.5, 2.5, -2.0, 0.7, 1.3])
    y = synthetic_y(9)
    a, b = weighted_per_level_ols(lv, z, y, np.ones(9), 4)
    checks = [[2, float(y[3:6].mean())]] + [[l, a[l]] for l in (0, 3)] + [[4 + l, b[l]] for l in (0, 3)]
    cases.append({"source": "tests/slopes.rs rank_drops_report_deterministically_with_exact_zeros",
                  "levels": lv.tolist(), "slopes": [z.tolist()], "y": [y.tolist()], "weights": None,
                  "drops": [[0, 1, 0], [0, 1, 1], [0, 2, 1]], "zero_slots": [1, 5, 6], "checks": checks,
                  "also_diagonal": True})
    # weighted_solve_matches_closed_form_and_masks_zero_weight_rows
    lv = np.array([0, 1, 0, 1, 0, 1, 2, 2, 2])
    z = np.array([0.5, -1.2, 3.3, 1.5, 0.7, -2.1, 5.0, 5.0, 7.0])
    w = np.array([1.0, 0.5, 2.0, 1.5, 3.0, 1.0, 1.0, 1.0, 0.0])
    y = synthetic_y(9)
    a, b = weighted_per_level_ols(lv, z, y, w, 3)
    checks = [[l, a[l]] for l in (0, 1)] + [[3 + l, b[l]] for l in (0, 1)] + [[2, float((y[6] + y[7]) / 2)]]
    cases.append({"source": "tests/slopes.rs weighted_solve_matches_closed_form_and_masks_zero_weight_rows",
                  "levels": lv.tolist(), "slopes": [z.tolist()], "y": [y.tolist()], "weights": w.tolist(),
                  "drops": [[0, 2, 1]], "zero_slots": [5], "checks": checks, "also_diagonal": False})
    # zero_weight_garbage_does_not_poison_identification
    lv = np.array([0, 0, 0, 1, 1, 1])
    z = np.array([1.0, 2.0, 3.0, 5.0, 7.0, 1e300])
    w = np.array([1.0, 1.0, 1.0, 1.0, 1.0, 0.0])
    y = synthetic_y(6)
    keep = w > 0
    a, b = weighted_per_level_ols(lv[keep], z[keep], y[keep], w[keep], 2)
    checks = [[l, a[l]] for l in (0, 1)] + [[2 + l, b[l]] for l in (0, 1)]
    cases.append({"source": "tests/slopes.rs zero_weight_garbage_does_not_poison_identification",
                  "levels": lv.tolist(), "slopes": [z.tolist()], "y": [y.tolist()], "weights": w.tolist(),
                  "drops": [], "zero_slots": [], "checks": checks, "also_diagonal": True})
    # batch_solve_shares_unidentified_and_back_transforms_each_rhs
    lv = np.array([0, 0, 0, 1, 1, 1])
    z = np.array([1.0, 2.0, 3.0, 2.5, 2.5, 2.5])
    y1 = synthetic_y(6)
    y2 = y1 * -1.5 + 0.3
    cases.append({"source": "tests/slopes.rs batch_solve_shares_unidentified_and_back_transforms_each_rhs",
                  "levels": lv.tolist(), "slopes": [z.tolist()], "y": [y1.tolist(), y2.tolist()],
                  "weights": None, "drops": [[0, 1, 1]], "zero_slots": [3], "checks": [],
                  "also_diagonal": False})
    # three_slopes_solve_bounded_with_exact_rank_drops: level 1's z2 and z3
    # are exactly collinear; the pivot keeps z3, so z2's slot reads 0
    n = 24
    lv = np.array([i % 3 for i in range(n)])
    z1 = np.array([math.sin(i * 0.37) * 2.0 for i in range(n)])
    z2 = np.array([0.95 * z1[i] + 0.1 * math.cos(i * 0.9 + 0.2) for i in range(n)])
    z3 = np.array([2.0 * z2[i] if i % 3 == 1 else -0.8 * z1[i] + 0.15 * math.sin(i * 1.7) + 0.1
                   for i in range(n)])
    y = synthetic_y(n)
    cases.append({"source": "tests/slopes.rs three_slopes_solve_bounded_with_exact_rank_drops",
                  "levels": lv.tolist(), "slopes": [z1.tolist(), z2.tolist(), z3.tolist()], "y": [y.tolist()],
                  "weights": None, "drops": [[0, 1, 2]], "zero_slots": [2 * 3 + 1], "checks": [],
                  "max_iterations": 30, "projection_tol": 1e-6, "also_diagonal": False})
    return cases


def lsmr_cases():
    """crates/schwarz-precond/src/lsmr/fixtures.rs and lsmr/tests/solve.rs."""
    over = [[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0]]
    rows, cols = 30, 12
    vand = [[(i / (rows - 1)) ** j for j in range(cols)] for i in range(rows)]
    vb = [math.log(1.0 + i / (rows - 1)) for i in range(rows)]
    jac = [1.0 / sum(vand[i][j] ** 2 for i in range(rows)) for j in range(cols)]
    return [
        {"source": "solve.rs test_mlsmr_unpreconditioned", "a": over, "b": [1, 2, 3, 3],
         "tol": 1e-10, "maxiter": 100, "x": [1, 2, 3], "x_tol": 1e-6},
        {"source": "solve.rs test_mlsmr_preconditioned", "a": over, "b": [1, 2, 3, 3],
         "tol": 1e-10, "maxiter": 100, "precond": [0.5, 0.5, 1.0], "x": [1, 2, 3], "x_tol": 1e-6},
        {"source": "solve.rs test_mlsmr_inconsistent_system", "a": over, "b": [1, 2, 3, 0],
         "tol": 1e-10, "maxiter": 100, "normal_eq_max": 1e-6},
        {"source": "solve.rs test_mlsmr_underdetermined_system", "a": [[1, 0, 0], [0, 1, 0]],
         "b": [1, 2], "tol": 1e-12, "maxiter": 100, "x": [1, 2, 0], "x_tol": 1e-10},
        {"source": "solve.rs test_lsmr_large_magnitude_rhs_not_silently_zero",
         "a": [[1, 0, 0], [0, 1, 0], [0, 0, 1]], "b": [1e155, 2e155, 3e155], "tol": 1e-10,
         "maxiter": 100, "x_rel": [1e155, 2e155, 3e155], "x_rel_tol": 1e-6},
        {"source": "solve.rs test_mlsmr_large_magnitude_rhs_not_silently_zero",
         "a": [[1, 0, 0], [0, 1, 0], [0, 0, 1]], "b": [1e155, 2e155, 3e155], "tol": 1e-10,
         "maxiter": 100, "precond": [1.0, 1.0, 1.0], "x_rel": [1e155, 2e155, 3e155], "x_rel_tol": 1e-6},
        {"source": "solve.rs test_mlsmr_local_reorth_unpreconditioned", "a": vand, "b": vb,
         "tol": 1e-9, "maxiter": 30, "local_size": 10, "normal_eq_max": 1e-6, "converged": True},
        {"source": "solve.rs test_mlsmr_local_reorth_preconditioned", "a": vand, "b": vb,
         "tol": 1e-9, "maxiter": 30, "local_size": 10, "precond": jac, "normal_eq_max": 1e-6,
         "converged": True},
        {"source": "solve.rs test_mlsmr_local_reorth_window_boundary_sizes (1)", "a": vand, "b": vb,
         "tol": 1e-9, "maxiter": 200, "local_size": 1, "normal_eq_max": 1e-6, "converged": True},
        {"source": "solve.rs test_mlsmr_local_reorth_window_boundary_sizes (12)", "a": vand, "b": vb,
         "tol": 1e-9, "maxiter": 200, "local_size": 12, "normal_eq_max": 1e-6, "converged": True},
        {"source": "solve.rs test_mlsmr_local_reorth_window_boundary_sizes (13)", "a": vand, "b": vb,
         "tol": 1e-9, "maxiter": 200, "local_size": 13, "normal_eq_max": 1e-6, "converged": True},
    ]


def main():
    out = {
        "stable_argsort": xorshift_keys(),
        "design": design_cases(),
        "slope_layout": slope_layout_case(),
        "level_means": {"source": "tests/metamorphic.rs:164-181",
                        "categories": [0, 0, 1, 1, 1, 2], "y": [1.0, 3.0, 2.0, 4.0, 6.0, 5.0],
                        "x": [2.0, 4.0, 5.0]},
        "slopes": slope_cases(),
        "slope_drops": slope_drop_cases(),
        "lsmr": lsmr_cases(),
        "vec_norm": {"source": "solve.rs vec_norm_is_overflow_safe_and_propagates_nan",
                     "cases": [[[], 0.0], [[3.0, 4.0], 5.0]]},
    }
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(out, f)
    print("wrote", os.path.join(HERE, "known_answers.json"))


if __name__ == "__main__":
    main()
