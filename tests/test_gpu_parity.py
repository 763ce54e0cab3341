"""GPU parity of the CUDA path against the CPU FP64 restatement (oracle).

Tolerances: demeaned vectors agree within 1e-7 in max|difference| / ||y||_2
(the contract's scaling, stated at tol 1e-8) and within 1e-6 in
max|difference| / max|y|; these tests solve tighter (tol 1e-10 to 1e-11) and
hold both bounds.  The contract tolerance itself, on the benchmark designs, is
tested in test_gpu_contract.py.  Integer work (grouping permutation, layout)
must match exactly.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import (as_solver_categories, demeaned_errors, dense_demeaned, generate_synthetic_data,
                      normal_equation_residual)

pytestmark = pytest.mark.gpu

DEMEAN_TOL = 1e-7        # max|difference| / ||y||_2
DEMEAN_TOL_INF = 1e-6    # max|difference| / max|y|


def rel_inf(a, b, y):
    """max|a - b| / ||y||_2, after checking max|a - b| / max|y| <= DEMEAN_TOL_INF."""
    e = demeaned_errors(a, b, y)
    assert e["inf_over_inf"] <= DEMEAN_TOL_INF, e
    return e["inf_over_l2"]


def two_factor(n=5000, l0=50, l1=30, seed=1):
    rng = np.random.default_rng(seed)
    cats = [rng.integers(0, l0, n), rng.integers(0, l1, n)]
    return cats, rng.standard_normal(n)


@pytest.mark.parametrize("kind", ["off", "diagonal", "additive"])
@pytest.mark.parametrize("weighted", [False, True])
def test_two_factor_matches_oracle(wb, oracle, kind, weighted):
    cats, y = two_factor()
    w = np.random.default_rng(7).lognormal(0, 1, len(y)) if weighted else None
    C = as_solver_categories(cats)
    pc = {"off": wb.PreconditionerConfig.Off, "diagonal": wb.PreconditionerConfig.Diagonal,
          "additive": wb.PreconditionerConfig.Additive}[kind]
    r = wb.solve(C, y, weights=w, options=wb.LsmrOptions(tol=1e-10, maxiter=5000), preconditioner=pc)
    o = oracle.OracleSolver(C, weights=w, cfg=oracle.precond_cfg(kind)).solve(y, tol=1e-10, maxiter=5000)
    assert r.converged and o.converged
    assert rel_inf(r.demeaned, o.demeaned, y) < DEMEAN_TOL
    assert rel_inf(r.demeaned, dense_demeaned(cats, y, w), y) < DEMEAN_TOL
    assert normal_equation_residual(cats, y, r.demeaned, w) < 1e-8


def test_three_factor_additive_matches_oracle(wb, oracle):
    rng = np.random.default_rng(3)
    n = 20000
    cats = [rng.integers(0, 400, n), rng.integers(0, 120, n), rng.integers(0, 15, n)]
    y = rng.standard_normal(n)
    C = as_solver_categories(cats)
    r = wb.solve(C, y, options=wb.LsmrOptions(tol=1e-10))
    o = oracle.OracleSolver(C).solve(y, tol=1e-10)
    assert r.converged
    assert rel_inf(r.demeaned, o.demeaned, y) < DEMEAN_TOL
    assert normal_equation_residual(cats, y, r.demeaned) < 1e-8


def test_slopes_weighted_matches_oracle(wb, oracle):
    rng = np.random.default_rng(5)
    n = 8000
    f = rng.integers(0, 60, n).astype(np.uint32)
    yr = rng.integers(0, 12, n).astype(np.uint32)
    z = rng.standard_normal(n)
    w = rng.lognormal(0, 0.5, n)
    y = rng.standard_normal(n)
    eff = [wb.Effect(f, True, [z]), wb.Effect(yr, True)]
    r = wb.solve(eff, y, weights=w, options=wb.LsmrOptions(tol=1e-11, maxiter=5000))
    o = oracle.OracleSolver([oracle.Effect(f, True, (z,)), oracle.Effect(yr, True)],
                            weights=w).solve(y, tol=1e-11, maxiter=5000)
    assert r.converged
    ref = dense_demeaned([f, yr], y, w, slopes=[(f, z)])
    assert rel_inf(r.demeaned, ref, y) < DEMEAN_TOL
    assert rel_inf(r.demeaned, o.demeaned, y) < DEMEAN_TOL


def test_grouping_and_layout_bit_exact(wb, oracle):
    """The locality-sort permutation and coefficient layout are integer
    results and must equal the restatement's exactly (domain.rs:187-247)."""
    rng = np.random.default_rng(11)
    n = 3000
    cats = [rng.integers(0, 40, n), rng.integers(0, 300, n), rng.integers(0, 7, n)]
    C = as_solver_categories(cats)
    s = wb.Solver(C, preconditioner=wb.PreconditionerConfig.Diagonal)
    o = oracle.OracleSolver(C, cfg=oracle.precond_cfg("diagonal"))
    np.testing.assert_array_equal(s.obs_perm(), o.obs_perm())
    for t in range(3):
        nl, off, nc, _ = o.term(t)
        assert (s.layout.n_levels(t), s.layout.n_columns(t)) == (nl, nc)
        assert s.layout.index(t, 0, 0) == off


def test_operator_apply_and_adjoint_match_oracle(wb, oracle):
    import torch
    rng = np.random.default_rng(13)
    n = 7000
    f = rng.integers(0, 90, n).astype(np.uint32)
    g = rng.integers(0, 25, n).astype(np.uint32)
    z = rng.standard_normal(n)
    w = rng.lognormal(0, 1, n)
    eff = [wb.Effect(f, True, [z]), wb.Effect(g, True)]
    s = wb.Solver(eff, weights=w, preconditioner=wb.PreconditionerConfig.Off)
    o = oracle.OracleSolver([oracle.Effect(f, True, (z,)), oracle.Effect(g, True)], weights=w,
                            cfg=oracle.precond_cfg("off"))
    x = rng.standard_normal(s.n_dofs)
    u = rng.standard_normal(n)
    xd = torch.tensor(x, device="cuda")
    ud = torch.tensor(u, device="cuda")
    ax = torch.empty(n, dtype=torch.float64, device="cuda")
    atu = torch.empty(s.n_dofs, dtype=torch.float64, device="cuda")
    s.operator_apply_device(xd, ax)
    s.operator_apply_adjoint_device(ud, atu)
    np.testing.assert_allclose(ax.cpu().numpy(), o.apply(x), rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(atu.cpu().numpy(), o.apply_adjoint(u), rtol=1e-12, atol=1e-11)


def test_schwarz_exact_route_matches_oracle(wb, oracle):
    """With kept blocks at or below dense_threshold both sides apply the exact
    local solves, so M^-1 r agrees to roundoff."""
    import torch
    rng = np.random.default_rng(17)
    n = 6000
    cats = [rng.integers(0, 200, n), rng.integers(0, 20, n), rng.integers(0, 12, n)]
    C = as_solver_categories(cats)
    s = wb.Solver(C)
    o = oracle.OracleSolver(C)
    p = s.preconditioner
    r = rng.standard_normal(s.n_dofs)
    rd = torch.tensor(r, device="cuda")
    zd = torch.empty_like(rd)
    p.apply_device(rd, zd)
    np.testing.assert_allclose(zd.cpu().numpy(), o.precond_apply(r), rtol=1e-9, atol=1e-10)


def test_schwarz_apply_symmetric_psd(wb):
    import torch
    rng = np.random.default_rng(19)
    n = 30000
    cats = [rng.integers(0, 3000, n), rng.integers(0, 400, n)]
    s = wb.Solver(as_solver_categories(cats))
    p = s.preconditioner
    a = torch.tensor(rng.standard_normal(s.n_dofs), device="cuda")
    b = torch.tensor(rng.standard_normal(s.n_dofs), device="cuda")
    ma, mb = torch.empty_like(a), torch.empty_like(b)
    p.apply_device(a, ma)
    p.apply_device(b, mb)
    lhs, rhs = float(ma @ b), float(a @ mb)
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), 1.0)
    assert float(ma @ a) >= 0.0


def test_solves_are_bitwise_reproducible(wb):
    cats, y = two_factor(n=20000, l0=700, l1=90, seed=23)
    s = wb.Solver(as_solver_categories(cats))
    a = s.solve(y)
    b = s.solve(y)
    assert a.iterations == b.iterations
    np.testing.assert_array_equal(a.demeaned, b.demeaned)
    np.testing.assert_array_equal(a.x, b.x)


@pytest.mark.parametrize("k", [2, 3, 8, 11])
def test_batch_matches_single(wb, k):
    cats, _ = two_factor(n=12000, l0=300, l1=40, seed=29)
    Y = np.random.default_rng(31).standard_normal((12000, k))
    s = wb.Solver(as_solver_categories(cats))
    opts = wb.LsmrOptions(tol=1e-11)
    b = s.solve_batch(Y, opts)
    assert b.demeaned.shape == (12000, k) and b.x.shape == (s.n_dofs, k)
    for j in range(k):
        r = s.solve(Y[:, j], opts)
        assert b.converged[j]
        assert rel_inf(b.demeaned[:, j], r.demeaned, Y[:, j]) < 1e-9


def test_known_answers(wb):
    # saturated single factor -> level means 2, 4, 5 (tests/metamorphic.rs:164-181)
    cats = np.array([[0], [0], [1], [1], [1], [2]], np.uint32)
    y = np.array([1.0, 3.0, 2.0, 4.0, 6.0, 5.0])
    r = wb.solve(np.asfortranarray(cats), y, options=wb.LsmrOptions(tol=1e-12))
    assert r.converged
    np.testing.assert_allclose(r.x[:3], [2.0, 4.0, 5.0], atol=1e-9)
    # noise-free y = D x_true -> demeaned == 0 (tests/conftest.py:7-21)
    cats2, _, y2 = generate_synthetic_data([50, 50], 10_000, seed=7)
    r2 = wb.solve(as_solver_categories(cats2), y2)
    assert r2.converged
    assert np.max(np.abs(r2.demeaned)) < 1e-6 * np.linalg.norm(y2)


def test_input_errors(wb):
    cats, y = two_factor(n=500, l0=10, l1=5)
    s = wb.Solver(as_solver_categories(cats))
    bad = y.copy()
    bad[3] = np.nan
    with pytest.raises(ValueError):
        s.solve(bad)
    with pytest.raises(ValueError):
        s.solve(y[:-1])
    w = np.ones_like(y)
    w[2] = -1.0
    with pytest.raises(ValueError):
        wb.Solver(as_solver_categories(cats), weights=w)
    with pytest.raises(TypeError):
        s.solve(y.astype(np.float32))


@pytest.mark.parametrize("path", ["0", "2"])
@pytest.mark.parametrize("seed", [0, 1])
def test_adjoint_sweep_classes_match_oracle(wb, oracle, seed, path, monkeypatch):
    """Both operator paths (WITHIN_SWEEP=0: gather plus segmented reduction,
    =2: warp-range row sweep) against the restatement's
    scatter: a worker-sorted term whose levels span many tiles and warp
    ranges, a firm term with runs along the worker order (and a slope), a
    12-level histogram term, weights, and an observation count that is not a
    multiple of any tile or chunk; single and 3-column solves go through the
    same path."""
    import torch
    monkeypatch.setenv("WITHIN_SWEEP", path)
    rng = np.random.default_rng(100 + seed)
    n_w = 300
    counts = rng.integers(1, 3000, n_w)
    worker = np.repeat(np.arange(n_w), counts).astype(np.uint32)
    n = worker.size
    firm = np.empty(n, np.uint32)
    cur = 0
    for i in range(n):
        if i == 0 or worker[i] != worker[i - 1] or rng.random() < 0.02:
            cur = rng.integers(0, 500)
        firm[i] = cur
    year = rng.integers(0, 12, n).astype(np.uint32)
    z = rng.standard_normal(n)
    w = rng.lognormal(0, 1, n)
    eff = [wb.Effect(worker, True), wb.Effect(firm, True, [z]), wb.Effect(year, True)]
    s = wb.Solver(eff, weights=w, preconditioner=wb.PreconditionerConfig.Diagonal)
    o = oracle.OracleSolver([oracle.Effect(worker, True), oracle.Effect(firm, True, (z,)),
                             oracle.Effect(year, True)], weights=w, cfg=oracle.precond_cfg("diagonal"))
    u = rng.standard_normal(n)
    ud = torch.tensor(u, device="cuda")
    atu = torch.empty(s.n_dofs, dtype=torch.float64, device="cuda")
    s.operator_apply_adjoint_device(ud, atu)
    np.testing.assert_allclose(atu.cpu().numpy(), o.apply_adjoint(u), rtol=1e-11, atol=1e-10)
    y = rng.standard_normal(n)
    r = s.solve(y, wb.LsmrOptions(tol=1e-10, maxiter=3000))
    ref = o.solve(y, tol=1e-10, maxiter=3000)
    assert r.converged
    assert rel_inf(r.demeaned, ref.demeaned, y) < DEMEAN_TOL
    Y = np.stack([y, z, rng.standard_normal(n)], axis=1)
    b = s.solve_batch(Y, wb.LsmrOptions(tol=1e-10, maxiter=3000))
    for k in range(3):
        refk = o.solve(np.ascontiguousarray(Y[:, k]), tol=1e-10, maxiter=3000)
        assert rel_inf(b.demeaned[:, k], refk.demeaned, Y[:, k]) < DEMEAN_TOL


@pytest.mark.parametrize("weighted", [False, True])
def test_intercept_sweep_multi_chunk_ranges(wb, oracle, weighted, monkeypatch):
    """The intercept-only row sweep on a panel long enough for several chunks
    per warp range (n > 3552 x 128): a worker-sorted term with some workers
    longer than a range, firm runs along the worker order (run ordinals, runs
    crossing chunks and ranges: the crossing-run fix-up launch), a 20-level
    histogram term, an observation count that is not a multiple of 4.  The
    adjoint against the restatement; solves against the gather + segmented
    reduction path (WITHIN_SWEEP=0)."""
    import torch
    rng = np.random.default_rng(5 + int(weighted))
    n_w = 60000
    counts = rng.integers(1, 40, n_w)
    counts[rng.choice(n_w, 20, replace=False)] = rng.integers(3000, 9000, 20)
    worker = np.repeat(np.arange(n_w), counts).astype(np.uint32)
    n = worker.size
    if n % 4 == 0:
        worker = worker[:-1]
        n -= 1
    change = np.ones(n, bool)
    change[1:] = (worker[1:] != worker[:-1]) | (rng.random(n - 1) < 0.03)
    firm = rng.integers(0, 8000, int(change.sum())).astype(np.uint32)[np.cumsum(change) - 1]
    year = rng.integers(0, 20, n).astype(np.uint32)
    cats = [worker, firm, year]
    w = rng.lognormal(0.0, 1.0, n) if weighted else None
    monkeypatch.delenv("WITHIN_SWEEP", raising=False)
    s = wb.Solver([wb.Effect(c, True) for c in cats], weights=w)
    o = oracle.OracleSolver([oracle.Effect(c, True) for c in cats], weights=w, cfg=oracle.precond_cfg("diagonal"))
    u = rng.standard_normal(n)
    atu = torch.empty(s.n_dofs, dtype=torch.float64, device="cuda")
    s.operator_apply_adjoint_device(torch.tensor(u, device="cuda"), atu)
    np.testing.assert_allclose(atu.cpu().numpy(), o.apply_adjoint(u), rtol=1e-11, atol=1e-9)
    y = rng.standard_normal(n)
    opts = wb.LsmrOptions(tol=1e-9, maxiter=5000)
    r = s.solve(y, opts)
    monkeypatch.setenv("WITHIN_SWEEP", "0")
    r0 = wb.Solver([wb.Effect(c, True) for c in cats], weights=w).solve(y, opts)
    assert r.converged and r0.converged
    assert abs(r.iterations - r0.iterations) <= 2, (r.iterations, r0.iterations)
    assert rel_inf(r.demeaned, r0.demeaned, y) < DEMEAN_TOL


@pytest.fixture(scope="module")
def multi_k_case(oracle):
    """A worker-sorted panel with a firm slope and a year term, weights, and 5
    right-hand sides with their restatement solutions."""
    rng = np.random.default_rng(77)
    n_w = 4000
    counts = rng.integers(1, 400, n_w)
    worker = np.repeat(np.arange(n_w), counts).astype(np.uint32)
    n = worker.size
    firm = np.empty(n, np.uint32)
    cur = 0
    for i in range(n):
        if i == 0 or worker[i] != worker[i - 1] or rng.random() < 0.05:
            cur = rng.integers(0, 3000)
        firm[i] = cur
    year = rng.integers(0, 30, n).astype(np.uint32)
    z = rng.standard_normal(n)
    w = rng.lognormal(0, 0.7, n)
    Y = np.asfortranarray(rng.standard_normal((n, 5)))
    o = oracle.OracleSolver([oracle.Effect(worker, True), oracle.Effect(firm, True, (z,)),
                             oracle.Effect(year, True)], weights=w, cfg=oracle.precond_cfg("diagonal"))
    refs = [o.solve(np.ascontiguousarray(Y[:, c]), tol=1e-11, maxiter=20000).demeaned for c in range(5)]
    return worker, firm, year, z, w, Y, refs


@pytest.mark.parametrize("path", ["0", "2"])
def test_every_column_bucket_on_every_path(wb, multi_k_case, path, monkeypatch):
    """Solves of 1, 2, 3 and 5 columns (the K = 1, 2, 4 and 8 kernels) on each
    operator path against the restatement, diagonal preconditioner."""
    monkeypatch.setenv("WITHIN_SWEEP", path)
    worker, firm, year, z, w, Y, refs = multi_k_case
    s = wb.Solver([wb.Effect(worker, True), wb.Effect(firm, True, [z]), wb.Effect(year, True)], weights=w,
                  preconditioner=wb.PreconditionerConfig.Diagonal)
    opts = wb.LsmrOptions(tol=1e-10, maxiter=20000)
    for k in (1, 2, 3, 5):
        b = s.solve_batch(np.asfortranarray(Y[:, :k]), opts)
        for c in range(k):
            assert b.converged[c]
            assert rel_inf(b.demeaned[:, c], refs[c], Y[:, c]) < DEMEAN_TOL, (k, c)


@pytest.mark.parametrize("local_size", [3, 10])
def test_windowed_reorthogonalisation_matches_restatement(wb, oracle, local_size):
    """local_size > 0: the M-orthogonal window (bidiag.rs:113-217, 489-512) on
    the GPU against the restatement's mlsmr with the same window, diagonal
    preconditioner (identical M): the same iteration count up to the drift
    of rounding over a long (~270 step) Krylov run (2 %), the same demeaned
    vector; single and 2-column solves."""
    rng = np.random.default_rng(31)
    n = 40_000
    worker = np.sort(rng.integers(0, 6000, n)).astype(np.uint32)
    firm = np.empty(n, np.uint32)
    cur = 0
    for i in range(n):
        if i == 0 or worker[i] != worker[i - 1] or rng.random() < 0.03:
            cur = rng.integers(0, 900)
        firm[i] = cur
    year = rng.integers(0, 15, n).astype(np.uint32)
    cats = [worker, firm, year]
    Y = np.asfortranarray(rng.standard_normal((n, 2)))
    s = wb.Solver(as_solver_categories(cats), preconditioner=wb.PreconditionerConfig.Diagonal)
    o = oracle.OracleSolver(as_solver_categories(cats), cfg=oracle.precond_cfg("diagonal"))
    opts = wb.LsmrOptions(tol=1e-10, maxiter=5000, local_size=local_size)
    b = s.solve_batch(Y, opts)
    for c in range(2):
        ref = o.solve(np.ascontiguousarray(Y[:, c]), tol=1e-10, maxiter=5000, local_size=local_size)
        assert b.converged[c]
        assert abs(b.iterations[c] - ref.iterations) <= max(2, 0.02 * ref.iterations), \
            (b.iterations[c], ref.iterations)
        assert rel_inf(b.demeaned[:, c], ref.demeaned, Y[:, c]) < DEMEAN_TOL
    r1 = s.solve(np.ascontiguousarray(Y[:, 0]), opts)
    assert abs(r1.iterations - b.iterations[0]) <= max(2, 0.02 * b.iterations[0])
    plain = s.solve(np.ascontiguousarray(Y[:, 0]), wb.LsmrOptions(tol=1e-10, maxiter=5000))
    assert rel_inf(r1.demeaned, plain.demeaned, Y[:, 0]) < DEMEAN_TOL


@pytest.mark.parametrize("tuning", [
    {"staged_sweep": 0},
    {"wide_mean_len": 32, "fuse_rounds": 0},
    {"wide_mean_len": 0xFFFFFFFF, "thread_per_segment": 0},
    {"core_small": 0, "core_min_frac": 0.1},
    {"core_dense_late": 256, "core_dense_max": 256},
    {"warp_ranges": 0},
    {"vector_rows": 1},
])
def test_tuning_records_match_oracle(wb, oracle, tuning):
    """Every kernel variant and factor rule a tuning record can select gives
    the oracle's demeaned vector: a worker-sorted panel (staged sweep, run and
    histogram terms, wide-tile plans, a round-scheduled factor with a fused
    tail) and a 3,000-level uniform design (its reduced system between the
    dense limits, which takes the small-graph rounds)."""
    from within_b200 import workloads as WL
    codes = WL.akm_panel(n=400_000, n_workers=40_000, n_firms=4_000, seed=21)
    y = np.random.default_rng(22).standard_normal(codes.shape[0])
    r = wb.Solver(codes, tuning=tuning).solve(y, wb.LsmrOptions(tol=1e-10, maxiter=3000))
    o = oracle.OracleSolver(codes).solve(y, tol=1e-10, maxiter=3000)
    assert r.converged
    assert rel_inf(r.demeaned, o.demeaned, y) < DEMEAN_TOL
    rng = np.random.default_rng(23)
    n = 150_000
    cats = [rng.integers(0, 20_000, n), rng.integers(0, 3_000, n), rng.integers(0, 12, n)]
    C = as_solver_categories(cats)
    y2 = rng.standard_normal(n)
    r2 = wb.Solver(C, tuning=tuning).solve(y2, wb.LsmrOptions(tol=1e-10, maxiter=3000))
    o2 = oracle.OracleSolver(C).solve(y2, tol=1e-10, maxiter=3000)
    assert r2.converged
    assert rel_inf(r2.demeaned, o2.demeaned, y2) < DEMEAN_TOL
