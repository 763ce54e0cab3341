"""Shared fixtures.  ``-m gpu`` tests need a CUDA device and the built
``within_b200/lib/libwithin_gpu.so``; everything else runs on the CPU."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def wb():
    """The product package; on a GPU box the library must load (no fallback)."""
    from within_b200 import _build
    _build.build()
    import within_b200
    return within_b200


def generate_synthetic_data(n_levels, n_rows, seed=42):
    """Noise-free y = D x_true (tests/conftest.py:7-21 of the reference)."""
    rng = np.random.default_rng(seed)
    cats = [rng.integers(0, nl, size=n_rows) for nl in n_levels]
    x_true = rng.standard_normal(sum(n_levels))
    y = np.zeros(n_rows)
    off = 0
    for f, nl in enumerate(n_levels):
        y += x_true[off + cats[f]]
        off += nl
    return cats, x_true, y


def as_solver_categories(cats):
    return np.asfortranarray(np.column_stack(cats).astype(np.uint32))


def normal_equation_residual(cats, y, demeaned, weights=None):
    """Independent optimality check ||D'W(y - Dx)|| / ||D'W y|| computed with
    bincount from the demeaned vector (tests/test_solve.py:23-44)."""
    y = np.asarray(y, np.float64)
    w = np.ones_like(y) if weights is None else np.asarray(weights, np.float64)
    num = den = 0.0
    for c in cats:
        c = np.asarray(c)
        num += np.square(np.bincount(c, weights=w * demeaned)).sum()
        den += np.square(np.bincount(c, weights=w * y)).sum()
    return num ** 0.5 / max(den ** 0.5, 1e-300)


def demeaned_errors(a, ref, y):
    """The difference of two demeaned vectors in both scalings the accuracy
    figures use: ``inf_over_inf`` = max|a - ref| / max|y| and
    ``inf_over_l2`` = max|a - ref| / ||y||_2.  The contract (1e-7 at tol
    1e-8) is stated on ``inf_over_l2``; on n rows of unit-scale data the
    second is about sqrt(n) / max|y| times smaller than the first."""
    d = float(np.max(np.abs(np.asarray(a) - np.asarray(ref)))) if np.size(a) else 0.0
    y = np.asarray(y)
    return {"inf_over_inf": d / max(float(np.max(np.abs(y))) if y.size else 0.0, 1e-300),
            "inf_over_l2": d / max(float(np.linalg.norm(y)), 1e-300)}


def check_slope_drop_case(case, x, demeaned, unidentified, iterations, y):
    """The expectations of one golden ``slope_drops`` case (tests/slopes.rs:157-326)
    on one solve: unidentified triples in ascending (level, column) order,
    exact zeros at the dropped slots, closed-form values (|got - exp| <=
    1e-6 (1 + |exp|), the reference's assert_close), and for the collinear
    case the iteration bound and residual orthogonality to every column of
    every level plus the fitted values."""
    assert [list(t) for t in unidentified] == case["drops"]
    for slot in case["zero_slots"]:
        assert x[slot] == 0.0, (slot, x[slot])
    assert np.all(np.isfinite(x))
    for slot, exp in case["checks"]:
        assert abs(x[slot] - exp) <= 1e-6 * (1 + abs(exp)), (slot, x[slot], exp)
    if "max_iterations" in case:
        assert iterations <= case["max_iterations"]
        lv = np.array(case["levels"])
        zs = [np.array(z) for z in case["slopes"]]
        nl = int(lv.max()) + 1
        for lvl in range(nl):
            m = lv == lvl
            for col in [None] + zs:
                dot = float(np.sum(demeaned[m] * (1.0 if col is None else col[m])))
                assert abs(dot) < case["projection_tol"], (lvl, dot)
        fitted = x[lv] + sum(x[(c + 1) * nl + lv] * zs[c] for c in range(len(zs)))
        exp = y - demeaned
        assert np.all(np.abs(fitted - exp) <= 1e-6 * (1 + np.abs(exp)))


def dense_demeaned(cats, y, weights=None, slopes=None):
    """Exact demeaned vector via dense least squares (small n only)."""
    n = len(y)
    cols = []
    for c in cats:
        c = np.asarray(c)
        L = int(c.max()) + 1
        M = np.zeros((n, L))
        M[np.arange(n), c] = 1.0
        cols.append(M)
    for (c, z) in (slopes or []):
        L = int(np.asarray(c).max()) + 1
        M = np.zeros((n, L))
        M[np.arange(n), c] = z
        cols.append(M)
    D = np.hstack(cols)
    sw = np.ones(n) if weights is None else np.sqrt(weights)
    x, *_ = np.linalg.lstsq(D * sw[:, None], y * sw, rcond=None)
    return y - D @ x
