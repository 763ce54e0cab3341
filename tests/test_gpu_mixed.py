"""Mixed precision (FP32 storage inside FP64 refinement on the normal-equation
residual): accuracy against the FP64 GPU solve at tol 1e-12 and against the
restatement, multi-RHS batches, weights, the diagonal preconditioner and the
stopping flags."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import normal_equation_residual

pytestmark = pytest.mark.gpu


def rel_inf(a, b, y):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(y)), 1e-300))


def panel(n, seed=5):
    from within_b200 import workloads as W
    codes = W.akm_panel(n=n, n_workers=max(1, n // 10), n_firms=max(1, n // 100), seed=seed)
    rng = np.random.default_rng(seed)
    return codes, rng.lognormal(0.0, 1.0, n)


@pytest.mark.parametrize("k", [1, 4])
def test_mixed_matches_fp64_oracle_solve(wb, k):
    """The mixed-precision accuracy target: at a tolerance where the plain FP64
    solve is within 1e-8 (max|d| / max|y|) of the FP64 solve at tol 1e-12
    (tol 1e-11: plain ~3e-10 on this panel), the mixed solve is too (measured
    ~5e-10 to 1.4e-9).  At the contract tolerance 1e-8 the two stopping tests
    stop at different points: the mixed solve's error was 1.2 to 4.6x the
    plain one's on this 300k-row panel (and below it on the 10M-row panel), so
    that case holds 10x, and the normal-equation residual (measured up to
    8x) 10x or 1e-6."""
    codes, w = panel(300_000)
    n = codes.shape[0]
    rng = np.random.default_rng(k)
    Y = np.asfortranarray(rng.standard_normal((n, k)))
    s64 = wb.Solver(codes, weights=w)
    ref = s64.solve_batch(Y, wb.LsmrOptions(tol=1e-12, maxiter=10000))
    smx = wb.Solver(codes, weights=w, precision="mixed")
    assert smx.precision == "mixed"
    cats = [codes[:, j] for j in range(3)]
    for tol in (1e-11, 1e-8):
        plain = s64.solve_batch(Y, wb.LsmrOptions(tol=tol))
        mx = smx.solve_batch(Y, wb.LsmrOptions(tol=tol))
        for c in range(k):
            assert mx.converged[c]
            e_mx = rel_inf(mx.demeaned[:, c], ref.demeaned[:, c], Y[:, c])
            e_plain = rel_inf(plain.demeaned[:, c], ref.demeaned[:, c], Y[:, c])
            if tol == 1e-11:
                assert e_plain <= 1e-8 and e_mx <= 1e-8, (e_mx, e_plain)
            else:
                assert e_mx <= 10.0 * e_plain, (e_mx, e_plain)
                ne_mx = normal_equation_residual(cats, Y[:, c], mx.demeaned[:, c], w)
                ne_plain = normal_equation_residual(cats, Y[:, c], plain.demeaned[:, c], w)
                assert ne_mx <= max(10.0 * ne_plain, 1e-6), (ne_mx, ne_plain)


def test_mixed_against_restatement_with_slopes_and_diagonal(wb, oracle):
    rng = np.random.default_rng(9)
    n = 60_000
    firm = rng.integers(0, 800, n).astype(np.uint32)
    year = rng.integers(0, 25, n).astype(np.uint32)
    z = rng.standard_normal(n)
    w = rng.lognormal(0.0, 0.5, n)
    y = rng.standard_normal(n)
    for kind, pc in (("additive", None), ("diagonal", wb.PreconditionerConfig.Diagonal)):
        s = wb.Solver([wb.Effect(firm, True, [z]), wb.Effect(year, True)], weights=w, preconditioner=pc,
                      precision="mixed")
        r = s.solve(y, wb.LsmrOptions(tol=1e-10, maxiter=20000))
        o = oracle.OracleSolver([oracle.Effect(firm, True, (z,)), oracle.Effect(year, True)], weights=w,
                                cfg=oracle.precond_cfg(kind, exact_local=True))
        ref = o.solve(y, tol=1e-12, maxiter=20000)
        assert r.converged, kind
        assert rel_inf(r.demeaned, ref.demeaned, y) < 1e-8, kind


def test_mixed_zero_and_fitted_columns(wb):
    codes, w = panel(50_000, seed=3)
    n = codes.shape[0]
    s = wb.Solver(codes, weights=w, precision="mixed")
    # column 0 zero, column 1 exactly in the span (demeaned = 0), column 2 noise
    x_true = np.random.default_rng(1).standard_normal(s.n_dofs)
    yfit = np.zeros(n)
    off = 0
    for j in range(3):
        L = int(codes[:, j].max()) + 1
        yfit += x_true[off + codes[:, j]]
        off += L
    Y = np.asfortranarray(np.column_stack([np.zeros(n), yfit, np.random.default_rng(2).standard_normal(n)]))
    b = s.solve_batch(Y, wb.LsmrOptions(tol=1e-8))
    assert all(b.converged)
    assert np.max(np.abs(b.demeaned[:, 0])) == 0.0
    assert np.max(np.abs(b.demeaned[:, 1])) / np.max(np.abs(yfit)) < 1e-7
    with pytest.raises(ValueError):
        s.set_precision("fp16")
