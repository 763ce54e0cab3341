"""Differentiable demeaning (torch.autograd.Function with the hand-written
adjoint): gradients with respect to z and the observation weights against an
explicit dense Jacobian, central finite differences (step 1e-6) and the
restatement solver applied to the adjoint right-hand side."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import dense_demeaned

pytestmark = pytest.mark.gpu


def pareto_codes(rng, n, n_levels, alpha=1.5):
    sizes = rng.pareto(alpha, n_levels) + 1.0
    p = sizes / sizes.sum()
    c = rng.choice(n_levels, size=n, p=p)
    # every level present, so n_levels = max + 1 and no empty level
    c[:n_levels] = np.arange(n_levels)
    return rng.permutation(c).astype(np.uint32)


def slopes_case(rng, n, n_firm, n_year):
    firm = pareto_codes(rng, n, n_firm)
    year = rng.integers(0, n_year, n).astype(np.uint32)
    year[:n_year] = np.arange(n_year)
    x = rng.standard_normal(n)
    w = rng.lognormal(0.0, 0.5, n)
    return firm, year, x, w


def dense_design(firm, year, x):
    n = firm.size
    Lf, Ly = int(firm.max()) + 1, int(year.max()) + 1
    D = np.zeros((n, 2 * Lf + Ly))
    D[np.arange(n), firm] = 1.0
    D[np.arange(n), Lf + firm] = x
    D[np.arange(n), 2 * Lf + year] = 1.0
    return D


def test_demean_gradients_match_dense_jacobian_and_fd(wb):
    import torch
    rng = np.random.default_rng(7)
    n = 1500
    firm, year, x, w = slopes_case(rng, n, 40, 8)
    eff = [wb.Effect(firm, True, [x]), wb.Effect(year, True)]
    z = rng.standard_normal((n, 2))
    v = rng.standard_normal((n, 2))
    opts = wb.LsmrOptions(tol=1e-13, maxiter=5000)
    zt = torch.tensor(z, device="cuda", requires_grad=True)
    wt = torch.tensor(w, device="cuda", requires_grad=True)
    out = wb.demean(zt, eff, weights=wt, options=opts)
    loss = (torch.tensor(v, device="cuda") * out).sum()
    loss.backward()
    gz = zt.grad.cpu().numpy()
    gw = wt.grad.cpu().numpy()

    # forward against dense least squares
    for c in range(2):
        ref = dense_demeaned([firm, year], z[:, c], w, slopes=[(firm, x)])
        assert np.max(np.abs(out[:, c].detach().cpu().numpy() - ref)) / np.max(np.abs(z[:, c])) < 1e-9

    # dL/dz = J^T v with J = I - D (D'WD)^+ D'W formed explicitly
    D = dense_design(firm, year, x)
    M = np.linalg.pinv(D.T @ (w[:, None] * D))
    J = np.eye(n) - D @ M @ (D.T * w[None, :])
    gz_ref = J.T @ v
    assert np.max(np.abs(gz - gz_ref)) / np.max(np.abs(gz_ref)) < 1e-9

    # dL/dw by central differences of the dense solution, 64 coordinates
    def dense_loss(wv):
        return sum(float(v[:, c] @ dense_demeaned([firm, year], z[:, c], wv, slopes=[(firm, x)]))
                   for c in range(2))
    h = 1e-6
    idx = rng.choice(n, 64, replace=False)
    fd = np.empty(idx.size)
    for j, i in enumerate(idx):
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd[j] = (dense_loss(wp) - dense_loss(wm)) / (2 * h)
    rel = np.max(np.abs(gw[idx] - fd)) / np.max(np.abs(fd))
    assert rel < 1e-5, rel


def test_demean_gradients_fd_through_gpu_solver_and_adjoint_rhs(wb, oracle):
    """Larger case: the weight gradient against central differences of the
    GPU solver itself (a new Solver per perturbed weight vector, tight
    tolerance), and the adjoint solve against the restatement."""
    import torch
    rng = np.random.default_rng(11)
    n = 40_000
    firm, year, x, w = slopes_case(rng, n, 2000, 30)
    eff = [wb.Effect(firm, True, [x]), wb.Effect(year, True)]
    z = rng.standard_normal(n)
    v = rng.standard_normal(n)
    opts = wb.LsmrOptions(tol=1e-13, maxiter=20000)
    zt = torch.tensor(z, device="cuda", requires_grad=True)
    wt = torch.tensor(w, device="cuda", requires_grad=True)
    out = wb.demean(zt, eff, weights=wt, options=opts)
    (torch.tensor(v, device="cuda") * out).sum().backward()
    gz = zt.grad.cpu().numpy()
    gw = wt.grad.cpu().numpy()

    # adjoint right-hand side through the restatement: dL/dz = w * demeaned(v / w)
    o = oracle.OracleSolver([oracle.Effect(firm, True, (x,)), oracle.Effect(year, True)], weights=w,
                            cfg=oracle.precond_cfg("additive", exact_local=True))
    s_ref = o.solve(v / w, tol=1e-12, maxiter=20000).demeaned
    assert np.max(np.abs(gz - w * s_ref)) / np.max(np.abs(w * s_ref)) < 1e-7

    def gpu_r(wv):
        s = wb.Solver(eff, weights=wv)
        return s.solve(z, opts).demeaned
    h = 1e-6
    idx = rng.choice(n, 16, replace=False)
    fd = np.empty(idx.size)
    for j, i in enumerate(idx):
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd[j] = float(v @ (gpu_r(wp) - gpu_r(wm))) / (2 * h)
    rel = np.max(np.abs(gw[idx] - fd)) / np.max(np.abs(fd))
    assert rel < 1e-5, rel


def test_demean_unweighted_and_vector_shapes(wb):
    import torch
    rng = np.random.default_rng(3)
    n = 5000
    a = rng.integers(0, 50, n).astype(np.uint32)
    b = rng.integers(0, 30, n).astype(np.uint32)
    cats = np.asfortranarray(np.column_stack([a, b]))
    z = rng.standard_normal(n)
    v = rng.standard_normal(n)
    zt = torch.tensor(z, device="cuda", requires_grad=True)
    out = wb.demean(zt, cats, options=wb.LsmrOptions(tol=1e-12, maxiter=5000))
    assert out.shape == (n,)
    (torch.tensor(v, device="cuda") * out).sum().backward()
    # unweighted: the Jacobian is the orthogonal projector, so dL/dz = demeaned(v)
    ref = dense_demeaned([a, b], v)
    assert np.max(np.abs(zt.grad.cpu().numpy() - ref)) / np.max(np.abs(ref)) < 1e-9
    with pytest.raises(ValueError):
        wb.demean(zt, cats, weights=torch.zeros(n, dtype=torch.float64, device="cuda"))
    with pytest.raises(TypeError):
        wb.demean(zt.float(), cats)


def test_demean_rejects_a_solver_built_with_other_weights(wb):
    """The forward solve uses the given solver's weights and the weight
    gradient the tensor passed to demean, so a mismatch must raise."""
    import torch
    rng = np.random.default_rng(5)
    n = 4000
    cats = np.asfortranarray(np.column_stack([rng.integers(0, 40, n), rng.integers(0, 25, n)]).astype(np.uint32))
    w = rng.lognormal(0.0, 0.5, n)
    zt = torch.tensor(rng.standard_normal(n), device="cuda", requires_grad=True)
    wt = torch.tensor(w, device="cuda", requires_grad=True)
    ok = wb.Solver(cats, weights=w)
    wb.demean(zt, cats, weights=wt, solver=ok)   # the same weights: accepted
    with pytest.raises(ValueError):
        wb.demean(zt, cats, weights=wt, solver=wb.Solver(cats, weights=w * 1.5))
    with pytest.raises(ValueError):
        wb.demean(zt, cats, weights=wt, solver=wb.Solver(cats))
    with pytest.raises(ValueError):
        wb.demean(zt, cats, solver=ok)
