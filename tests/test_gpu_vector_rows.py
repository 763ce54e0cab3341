"""The C back-substitution's rows by groups of lanes (within_tuning
vector_rows = 1, segvec_kernel) against one thread per row: every column
bucket in FP64, the mixed-precision solve (FP32 sums), run-to-run bitwise
reproducibility, and the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import demeaned_errors

pytestmark = pytest.mark.gpu

VR = {"vector_rows": 1}


def _panel(n, seed):
    from within_b200 import workloads as WL
    return WL.akm_panel(n=n, n_workers=n // 10, n_firms=n // 100, seed=seed)


def test_vector_rows_match_oracle(wb, oracle):
    codes = _panel(300_000, 61)
    y = np.random.default_rng(62).standard_normal(codes.shape[0])
    r = wb.Solver(codes, tuning=VR).solve(y, wb.LsmrOptions(tol=1e-10, maxiter=3000))
    o = oracle.OracleSolver(codes).solve(y, tol=1e-10, maxiter=3000)
    assert r.converged
    e = demeaned_errors(r.demeaned, o.demeaned, y)
    assert e["inf_over_l2"] < 1e-7 and e["inf_over_inf"] < 1e-6, e


@pytest.mark.parametrize("k", [2, 4, 8])
def test_vector_rows_batched_match_thread_rows(wb, k):
    codes = _panel(200_000, 63)
    Y = np.asfortranarray(np.random.default_rng(64).standard_normal((codes.shape[0], k)))
    opts = wb.LsmrOptions(tol=1e-11, maxiter=3000)
    a = wb.Solver(codes, tuning={"vector_rows": 0}).solve_batch(Y, opts)
    b = wb.Solver(codes, tuning=VR).solve_batch(Y, opts)
    for j in range(k):
        e = demeaned_errors(b.demeaned[:, j], a.demeaned[:, j], Y[:, j])
        assert e["inf_over_l2"] < 1e-8 and e["inf_over_inf"] < 1e-6, e


def test_vector_rows_mixed_precision(wb):
    codes = _panel(300_000, 65)
    rng = np.random.default_rng(66)
    w = rng.lognormal(0.0, 1.0, codes.shape[0])
    Y = np.asfortranarray(rng.standard_normal((codes.shape[0], 4)))
    ref = wb.Solver(codes, weights=w).solve_batch(Y, wb.LsmrOptions(tol=1e-12, maxiter=5000))
    mx = wb.Solver(codes, weights=w, precision="mixed", tuning=VR).solve_batch(Y, wb.LsmrOptions(tol=1e-11,
                                                                                                 maxiter=5000))
    for j in range(4):
        assert mx.converged[j]
        d = np.max(np.abs(mx.demeaned[:, j] - ref.demeaned[:, j]))
        assert d / np.max(np.abs(Y[:, j])) < 1e-8


def test_vector_rows_bitwise_reproducible(wb):
    codes = _panel(250_000, 67)
    y = np.random.default_rng(68).standard_normal(codes.shape[0])
    opts = wb.LsmrOptions(tol=1e-9)
    a = wb.Solver(codes, tuning=VR).solve(y, opts)
    b = wb.Solver(codes, tuning=VR).solve(y, opts)
    assert np.array_equal(a.demeaned, b.demeaned) and np.array_equal(a.x, b.x)
