"""Warm starts and escalation on the GPU (crates/schwarz-precond/src/lsmr.rs:
83-171, the reference's lsmr/tests/ladder.rs), through
within_solver_solve_batch_device_ext.

- A warm start from an iterate near the solution takes fewer iterations than
  a cold solve, its tolerance stays relative to the original ||b||, and it
  lands on the same demeaned vector; an exact warm start returns x0 untouched
  after 0 iterations (WarmStartExact); a zero right-hand side with a non-zero
  warm start corrects it back to the solution.
- Non-finite warm starts and staleness thresholds outside [0, 1) are input
  errors; a warm start on a slope design is refused.
- The staleness rule ends a stalling column with Escalated and hands its
  iterate to the next rung; the two-rung ladder (diagonal, then additive
  Schwarz warm-started) reaches the cold additive solve's demeaned vector.
- A converged column is never reported Escalated.
Tolerances as in test_gpu_parity.py (1e-7 of ||y||_2, 1e-6 of max|y|).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import as_solver_categories, demeaned_errors

pytestmark = pytest.mark.gpu


def panel(n=200_000, seed=9):
    from within_b200 import workloads as WL
    codes = WL.akm_panel(n=n, n_workers=n // 10, n_firms=n // 100, seed=seed)
    y = np.random.default_rng(seed).standard_normal(n)
    return codes, y


def close(a, b, y):
    e = demeaned_errors(a, b, y)
    assert e["inf_over_l2"] <= 1e-7 and e["inf_over_inf"] <= 1e-6, e


def test_warm_start_is_shorter_and_lands_on_the_cold_solution(wb):
    import torch
    codes, y = panel()
    s = wb.Solver(codes)
    yd = torch.tensor(y, device="cuda")
    opts = wb.LsmrOptions(tol=1e-10, maxiter=2000)
    cold = s.mlsmr_device(yd, opts)
    assert cold.converged[0] and cold.stop_reason[0] in ("NormalEquationTolerance", "ResidualTolerance")
    x0 = cold.x[:, 0] * (1 - 1e-4)
    warm = s.mlsmr_device(yd, opts, warm_start=x0)
    assert warm.converged[0]
    assert warm.iterations[0] < cold.iterations[0], (warm.iterations, cold.iterations)
    close(warm.demeaned[:, 0].cpu().numpy(), cold.demeaned[:, 0].cpu().numpy(), y)


def test_exact_and_zero_rhs_warm_starts(wb):
    import torch
    rng = np.random.default_rng(3)
    n = 20_000
    cats = [rng.integers(0, 300, n), rng.integers(0, 40, n)]
    s = wb.Solver(as_solver_categories(cats))
    # y exactly in the span: y = D x_true, warm start x_true -> b - A x0 = 0 exactly
    x_true = np.round(rng.standard_normal(s.n_dofs) * 8) / 8     # dyadic: D x is exact in FP64
    off1 = s.layout.index(1, 0, 0)
    y = x_true[cats[0]] + x_true[off1 + cats[1]]
    yd = torch.tensor(y, device="cuda")
    x0 = torch.tensor(x_true, device="cuda")
    r = s.mlsmr_device(yd, wb.LsmrOptions(tol=1e-10), warm_start=x0)
    assert r.stop_reason[0] == "WarmStartExact" and r.converged[0] and r.iterations[0] == 0
    assert torch.equal(r.x[:, 0], x0)
    assert float(r.demeaned.abs().max()) == 0.0
    # zero rhs, non-zero warm start: corrected towards the zero solution's
    # demeaned vector (0); the tolerance is relative to ||b|| = 0, so only the
    # residual shrinking is asserted, not a convergence flag
    z = torch.zeros(n, dtype=torch.float64, device="cuda")
    r0 = s.mlsmr_device(z, wb.LsmrOptions(tol=1e-14, maxiter=300), warm_start=x0)
    assert r0.iterations[0] > 0
    assert float(r0.demeaned.abs().max()) < 1e-8 * float(np.abs(y).max())


def test_warm_start_and_escalation_input_errors(wb):
    import torch
    rng = np.random.default_rng(4)
    n = 5_000
    cats = [rng.integers(0, 100, n), rng.integers(0, 20, n)]
    s = wb.Solver(as_solver_categories(cats))
    yd = torch.tensor(rng.standard_normal(n), device="cuda")
    bad = torch.zeros(s.n_dofs, dtype=torch.float64, device="cuda")
    bad[7] = float("nan")
    with pytest.raises(ValueError):
        s.mlsmr_device(yd, None, warm_start=bad)
    with pytest.raises(ValueError):
        s.mlsmr_device(yd, None, warm_start=torch.zeros(s.n_dofs - 1, dtype=torch.float64, device="cuda"))
    with pytest.raises(ValueError):
        wb.Staleness(0, 0.5)
    with pytest.raises(ValueError):
        wb.Staleness(3, 1.0)
    huge = torch.full((s.n_dofs,), 1e308, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):   # b - A x0 overflows: non-finite residual norm
        s.mlsmr_device(yd, None, warm_start=huge)
    f = rng.integers(0, 50, n).astype(np.uint32)
    sl = wb.Solver([wb.Effect(f, True, [rng.standard_normal(n)])])
    with pytest.raises(RuntimeError):
        sl.mlsmr_device(yd, None, warm_start=torch.zeros(sl.n_dofs, dtype=torch.float64, device="cuda"))


def test_staleness_escalates_and_ladder_matches_cold_solve(wb):
    import torch
    codes, y = panel(seed=11)
    Y = np.asfortranarray(np.column_stack([y, np.random.default_rng(12).standard_normal(y.size)]))
    opts = wb.LsmrOptions(tol=1e-10, maxiter=3000)
    weak = wb.Solver(codes, preconditioner=wb.PreconditionerConfig.Diagonal)
    Yd = torch.tensor(Y, device="cuda").t().contiguous().t()
    esc = weak.mlsmr_device(Yd, opts, escalation=wb.Staleness(2, 0.2))
    assert all(r == "Escalated" for r in esc.stop_reason), esc.stop_reason
    assert not any(esc.converged)
    lad = wb.solve_ladder(codes, Y, options=opts, escalation=wb.Staleness(2, 0.2))
    assert lad.rung == ["Additive", "Additive"] and all(lad.converged)
    cold = wb.Solver(codes).solve_batch(Y, opts)
    for j in range(2):
        close(lad.demeaned[:, j], cold.demeaned[:, j], Y[:, j])
    # a lenient rule lets the diagonal rung finish: converged, never Escalated
    easy = weak.mlsmr_device(Yd[:, :1], wb.LsmrOptions(tol=1e-6, maxiter=3000), escalation=wb.Staleness(500, 0.999))
    assert easy.converged[0] and easy.stop_reason[0] != "Escalated"
