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
