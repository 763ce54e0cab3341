"""The allocation-free adjoint entry point against the existing one.

within_solver_operator_apply_adjoint_noalloc exists for callers that cannot
allocate device memory during a call (stream capture, runtimes owning all
device memory, latency-critical paths); its scratch is a static device array
shared by every call.  Two calls in a row must each reproduce the existing
entry point's result on their own input, which also shows that the state the
first call leaves in the shared array does not leak into the second.  This
file is collected last so that a failure here comes after every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_adjoint_matches_existing_two_calls(wb):
    import torch
    from within_b200 import _ffi
    L = _ffi.lib()
    rng = np.random.default_rng(41)
    n = 300_000
    sizes = rng.pareto(1.5, 2_000) + 1.0
    firm = np.minimum(np.searchsorted(np.cumsum(sizes / sizes.sum()), rng.random(n)), 1_999)
    cats = np.asfortranarray(np.column_stack([rng.integers(0, 30_000, n), firm,
                                              rng.integers(0, 12, n)]).astype(np.uint32))
    w = rng.lognormal(0.0, 1.0, n)
    s = wb.Solver(cats, weights=w, preconditioner=wb.PreconditionerConfig.Diagonal)
    nd = s.n_dofs
    for call in range(2):
        u = torch.tensor(rng.standard_normal(n), device="cuda")
        torch.cuda.synchronize()   # the copy ran on torch's stream, the calls use the solver's
        ref = torch.empty(nd, dtype=torch.float64, device="cuda")
        s.operator_apply_adjoint_device(u, ref)
        out = torch.full((nd,), float("nan"), dtype=torch.float64, device="cuda")
        _ffi.check(L.within_solver_operator_apply_adjoint_noalloc(
            s.handle, C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr()), None))
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=1e-12, atol=1e-12)


def test_noalloc_adjoint_on_callers_stream_and_on_a_fresh_solver(wb):
    """On a fresh solver (no solve or adjoint call yet: the single-column plan
    is built at construction) and on the caller's own stream (torch's current
    stream, no wait inside the call) it matches the existing entry point."""
    import torch
    from within_b200 import _ffi
    L = _ffi.lib()
    rng = np.random.default_rng(43)
    n = 50_000
    cats = np.asfortranarray(np.column_stack([rng.integers(0, 4_000, n), rng.integers(0, 300, n)])
                             .astype(np.uint32))
    for pc in (wb.PreconditionerConfig.Diagonal, wb.PreconditionerConfig.Off):
        fresh = wb.Solver(cats, preconditioner=pc)
        u = torch.tensor(rng.standard_normal(n), device="cuda")
        out = torch.full((fresh.n_dofs,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        _ffi.check(L.within_solver_operator_apply_adjoint_noalloc(fresh.handle, C.c_void_p(u.data_ptr()),
                                                                  C.c_void_p(out.data_ptr()), None))
        first = out.cpu().numpy()
        ref = torch.empty_like(out)
        fresh.operator_apply_adjoint_device(u, ref)
        torch.cuda.synchronize()
        np.testing.assert_allclose(first, ref.cpu().numpy(), rtol=1e-12, atol=1e-12)
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            for _ in range(2):
                out.fill_(float("nan"))
                _ffi.check(L.within_solver_operator_apply_adjoint_noalloc(
                    fresh.handle, C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr()),
                    C.c_void_p(stream.cuda_stream)))
                stream.synchronize()
                np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=1e-12, atol=1e-12)
