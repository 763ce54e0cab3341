"""Seeded synthetic designs with the shapes of the solve benchmarks.

No public dataset is involved anywhere: each generator draws codes, weights
and responses from ``numpy.random.default_rng(seed)``.

- ``small_two_factor``  n = 100,000; codes uniform in [0,500) and [0,200).
- ``akm_panel``         n = 10,000,000 worker/firm/year panel: 1,000,000
  workers with geometric(mean 10) observation counts (the row count is
  truncated/padded to exactly n), 100,000 firms with Pareto(alpha = 1.5)
  sizes, each worker starting at a firm drawn in proportion to size and
  switching with probability 0.1 per observation, year uniform over 20.
- ``many_designs``      independent designs, n log-uniform in [1e4, 2e6],
  2 or 3 factors with level counts log-uniform in [20, n/10].
- ``slopes_panel``      n = 2,000,000; firm (50,000 Pareto(1.5) sizes) with an
  intercept and a slope on x ~ N(0,1), year (30 levels) intercept.
- ``fixest_like``       the reference's wall-clock DGP shape
  (crates/within/benches/shared/fixest_dgp.rs): 10 observations per worker,
  ~23 workers per firm, ``i % n_firm`` firms in the "difficult" variant.
"""
from __future__ import annotations

import numpy as np


def small_two_factor(n=100_000, seed=1):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 500, n).astype(np.uint32)
    b = rng.integers(0, 200, n).astype(np.uint32)
    y = rng.standard_normal(n)
    return np.asfortranarray(np.column_stack([a, b])), y


def _pareto_sizes(rng, n, alpha):
    return rng.pareto(alpha, n) + 1.0


def akm_panel(n=10_000_000, n_workers=1_000_000, n_firms=100_000, n_years=20, p_switch=0.1,
              alpha=1.5, seed=2):
    """Worker-sorted rows (worker codes non-decreasing)."""
    rng = np.random.default_rng(seed)
    counts = rng.geometric(1.0 / 10.0, n_workers)
    ends = np.cumsum(counts)
    worker = np.searchsorted(ends, np.arange(n), side="right")
    np.minimum(worker, n_workers - 1, out=worker)
    worker = worker.astype(np.uint32)
    first = np.ones(n, dtype=bool)
    first[1:] = worker[1:] != worker[:-1]
    switch = first | (rng.random(n) < p_switch)
    idx = np.flatnonzero(switch)
    sizes = _pareto_sizes(rng, n_firms, alpha)
    cdf = np.cumsum(sizes / sizes.sum())
    draws = np.searchsorted(cdf, rng.random(idx.size), side="right")
    np.minimum(draws, n_firms - 1, out=draws)
    last_switch = np.maximum.accumulate(np.where(switch, np.arange(n), 0))
    pos = np.searchsorted(idx, last_switch)
    firm = draws[pos].astype(np.uint32)
    year = rng.integers(0, n_years, n).astype(np.uint32)
    codes = np.asfortranarray(np.column_stack([worker, firm, year]))
    return codes


def akm_response(n, k=1, seed=12):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, k)) if k > 1 else rng.standard_normal(n)


def lognormal_weights(n, sigma=1.0, seed=22):
    return np.random.default_rng(seed).lognormal(0.0, sigma, n)


def many_designs(count=256, lo=10_000, hi=2_000_000, k=8, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        q = int(rng.integers(2, 4))
        cols = []
        for _ in range(q):
            L = int(np.exp(rng.uniform(np.log(20), np.log(max(21, n / 10)))))
            cols.append(rng.integers(0, L, n).astype(np.uint32))
        Y = rng.standard_normal((n, k))
        out.append((np.asfortranarray(np.column_stack(cols)), np.asfortranarray(Y)))
    return out


def slopes_panel(n=2_000_000, n_firms=50_000, n_years=30, alpha=1.5, seed=5):
    rng = np.random.default_rng(seed)
    sizes = _pareto_sizes(rng, n_firms, alpha)
    cdf = np.cumsum(sizes / sizes.sum())
    firm = np.minimum(np.searchsorted(cdf, rng.random(n), side="right"), n_firms - 1).astype(np.uint32)
    year = rng.integers(0, n_years, n).astype(np.uint32)
    x = rng.standard_normal(n)
    z = rng.standard_normal(n)
    w = rng.lognormal(0.0, 0.5, n)
    v = rng.standard_normal(n)
    return firm, year, x, z, w, v


def fixest_like(n=1_000_000, n_fe=3, difficult=True, seed=42):
    rng = np.random.default_rng(seed)
    n_years, per_firm = 10, 23
    n_indiv = max(1, round(n / n_years))
    n_firm = max(1, round(n_indiv / per_firm))
    i = np.arange(n)
    indiv = (i // n_years).astype(np.uint32)
    year = (i % n_years).astype(np.uint32)
    firm = (i % n_firm if difficult else rng.integers(0, n_firm, n)).astype(np.uint32)
    cols = [indiv, year] if n_fe == 2 else [indiv, year, firm]
    y = rng.uniform(-1.0, 1.0, n)
    return np.asfortranarray(np.column_stack(cols)), y
