"""Persisted preconditioner (pickling, crates/within-py/src/config.rs:366-389)
and the FWL regression step (README.md:54-65 of the reference).

- A Schwarz preconditioner serialised, read back and used as the prebuilt
  preconditioner of a new Solver gives solves bitwise equal to the original
  solver's; the same through pickle and for the diagonal variant.
- Corrupt, truncated or foreign bytes are rejected (ValueError), and a
  prebuilt preconditioner of another DOF count is refused.
- fwl: beta of the regression of y on X with the fixed effects absorbed,
  against numpy lstsq on the oracle's demeaned columns (rtol 1e-8), weighted
  and unweighted.
"""
from __future__ import annotations

import pickle

import numpy as np
import pytest

from conftest import as_solver_categories

pytestmark = pytest.mark.gpu


def design(seed=3, n=40_000):
    rng = np.random.default_rng(seed)
    cats = [rng.integers(0, 900, n), rng.integers(0, 150, n), rng.integers(0, 12, n)]
    return as_solver_categories(cats), rng.standard_normal(n)


def test_schwarz_preconditioner_round_trip_is_bitwise(wb):
    C, y = design()
    s = wb.Solver(C)
    p = s.preconditioner
    assert p.variant_name == "Additive"
    data = p.to_bytes()
    p2 = wb.Preconditioner.from_bytes(data)
    assert p2.nrows() == p.nrows() and p2.variant_name == "Additive"
    assert p2.to_bytes() == data
    s2 = wb.Solver(C, preconditioner=p2)
    a, b = s.solve(y), s2.solve(y)
    assert a.iterations == b.iterations
    np.testing.assert_array_equal(a.demeaned, b.demeaned)
    np.testing.assert_array_equal(a.x, b.x)
    p3 = pickle.loads(pickle.dumps(p))
    c = wb.Solver(C, preconditioner=p3).solve(y)
    np.testing.assert_array_equal(a.demeaned, c.demeaned)


def test_diagonal_preconditioner_round_trip(wb):
    C, y = design(seed=5)
    s = wb.Solver(C, preconditioner=wb.PreconditionerConfig.Diagonal)
    p = s.preconditioner
    assert p.variant_name == "Diagonal"
    p2 = pickle.loads(pickle.dumps(p))
    a = s.solve(y)
    b = wb.Solver(C, preconditioner=p2).solve(y)
    np.testing.assert_array_equal(a.demeaned, b.demeaned)


def test_bad_bytes_and_shape_mismatch_are_rejected(wb):
    C, _ = design(seed=7, n=5_000)
    data = wb.Solver(C).preconditioner.to_bytes()
    bad = bytearray(data)
    bad[len(bad) // 2] ^= 0xFF
    for blob in (bytes(bad), data[:-9], b"not a preconditioner at all", b""):
        with pytest.raises(ValueError):
            wb.Preconditioner.from_bytes(blob)
    other, _ = design(seed=8, n=5_000)
    other = other[:, :2].copy(order="F")
    p = wb.Preconditioner.from_bytes(data)
    with pytest.raises(ValueError):
        wb.Solver(other, preconditioner=p)


@pytest.mark.parametrize("weighted", [False, True])
def test_fwl_matches_lstsq_on_oracle_demeaned(wb, oracle, weighted):
    rng = np.random.default_rng(11)
    n = 60_000
    fe = np.asfortranarray(np.column_stack([rng.integers(0, 500, n), rng.integers(0, 200, n)])
                           .astype(np.uint32))
    beta_true = np.array([1.0, -2.0, 0.5])
    X = rng.standard_normal((n, 3))
    y = X @ beta_true + rng.standard_normal(n)
    w = rng.lognormal(0.0, 0.5, n) if weighted else None
    opts = wb.LsmrOptions(tol=1e-11, maxiter=5000)
    r = wb.fwl(fe, y, X, weights=w, options=opts)
    assert all(r.converged)
    o = oracle.OracleSolver(fe, weights=w)
    cols = [o.solve(np.ascontiguousarray(c), tol=1e-12, maxiter=5000).demeaned for c in [y, *X.T]]
    sw = np.ones(n) if w is None else np.sqrt(w)
    ref = np.linalg.lstsq(np.column_stack(cols[1:]) * sw[:, None], cols[0] * sw, rcond=None)[0]
    np.testing.assert_allclose(r.beta, ref, rtol=1e-8, atol=1e-10)
    assert np.max(np.abs(r.beta - beta_true)) < 0.05
