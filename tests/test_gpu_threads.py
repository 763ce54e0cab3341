"""Concurrent calls through the C ABI (tests/test_free_threaded.py:32-58 of
the reference): one Solver shared by several host threads, and one Solver per
thread.  ctypes drops the GIL for every call, so the calls really are
concurrent on the host.  Calls on one handle are serialised by the solver's
mutex, so every result equals the serial one bit for bit; separate solvers
share nothing but the device and run side by side on their own streams."""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor
from threading import Barrier

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_shared_solver_handles_parallel_solves(wb):
    rng = np.random.default_rng(42)
    categories = np.asfortranarray(rng.integers(0, 32, size=(4_096, 3), dtype=np.uint32))
    y = rng.standard_normal(categories.shape[0])
    y.setflags(write=False)
    solver = wb.Solver(categories)
    expected = solver.solve(y)
    assert expected.converged
    barrier = Barrier(4)

    def solve(_):
        barrier.wait()
        r = solver.solve(y)
        assert r.converged
        return r.x, r.demeaned

    with ThreadPoolExecutor(max_workers=4) as ex:
        results = list(ex.map(solve, range(16)))
    for x, dm in results:
        np.testing.assert_array_equal(x, expected.x)
        np.testing.assert_array_equal(dm, expected.demeaned)


def test_solver_per_thread_and_mixed_calls(wb):
    """Four solvers of different designs on four threads, each thread also
    calling solve_batch and the adjoint on its own solver."""
    import torch
    rng = np.random.default_rng(7)
    designs = [np.asfortranarray(rng.integers(0, L, size=(60_000, 2), dtype=np.uint32)) for L in (50, 400, 2000, 9000)]
    Ys = [np.asfortranarray(rng.standard_normal((60_000, 3))) for _ in designs]
    solvers = [wb.Solver(d) for d in designs]
    opts = wb.LsmrOptions(tol=1e-10)
    expected = [s.solve_batch(Y, opts) for s, Y in zip(solvers, Ys)]
    u = rng.standard_normal(60_000)
    def on_device(a):   # the copy is on torch's stream; the solver runs on its own
        t = torch.tensor(a, device="cuda")
        torch.cuda.current_stream().synchronize()
        return t

    adj = []
    for s in solvers:
        out = torch.empty(s.n_dofs, dtype=torch.float64, device="cuda")
        s.operator_apply_adjoint_device(on_device(u), out)
        adj.append(out.cpu().numpy())
    barrier = Barrier(4)

    def work(i):
        barrier.wait()
        s = solvers[i]
        got = []
        for _ in range(3):
            b = s.solve_batch(Ys[i], opts)
            out = torch.empty(s.n_dofs, dtype=torch.float64, device="cuda")
            s.operator_apply_adjoint_device(on_device(u), out)
            got.append((b.demeaned, out.cpu().numpy()))
        return got

    with ThreadPoolExecutor(max_workers=4) as ex:
        results = list(ex.map(work, range(4)))
    for i, got in enumerate(results):
        for dm, a in got:
            np.testing.assert_array_equal(dm, expected[i].demeaned)
            np.testing.assert_array_equal(a, adj[i])
