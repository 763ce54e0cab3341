"""Differentiable demeaning: ``demean(z, design, weights)`` = z - D x*(z, w)
as a ``torch.autograd.Function`` with a hand-written adjoint.

The forward is ``Solver.solve`` on device buffers (demeaned = y - D x,
crates/within/src/solver.rs:468-473).  For a loss gradient v on the output r,
with M the pseudo-inverse of D'WD:

    dL/dz = v - W D M D' v = w * demeaned(v / w)
    dL/dw = -r * (D M D' v) = -r * (a - demeaned(a)),   a = v / w

so the backward pass is one more preconditioned solve with the same
operator, weights and cached factors (the same ``Solver``), bracketed by two
per-observation CUDA kernels (``within_adjoint_rhs``, ``within_demean_vjp``;
the second fuses the forward and adjoint residuals into the weight
gradient).  Weights must be positive for dL/dw.  Everything runs on the GPU
through ``libwithin_gpu.so``; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi


def _colmajor(t):
    """(n,) -> (n, 1); (n, k) -> column-major (n, k) view of a contiguous copy."""
    if t.dim() == 1:
        return t.reshape(-1, 1)
    return t if t.stride(0) == 1 and t.stride(1) == t.shape[0] else t.t().contiguous().t()


def _stream(dev):
    import torch
    # torch's default stream (handle 0) is passed as cudaStreamLegacy: NULL
    # would select the solver's own stream, unordered with torch's work
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream or _ffi.CUDA_STREAM_LEGACY)


def _check_f64_cuda(name, t):
    import torch
    if not isinstance(t, torch.Tensor) or t.dtype != torch.float64 or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA float64 tensor")


class DemeanFunction:
    """Namespace holding the autograd Function (built lazily so importing the
    package does not import torch)."""
    _fn = None

    @classmethod
    def get(cls):
        if cls._fn is not None:
            return cls._fn
        import torch

        class _Demean(torch.autograd.Function):
            @staticmethod
            def forward(ctx, z, weights, solver, options):
                Z = _colmajor(z.detach())
                _, D, stats = solver.solve_device(Z, options)
                ctx.solver = solver
                ctx.options = options
                ctx.shape = z.shape
                ctx.has_w = weights is not None
                ctx.stats = stats
                ctx.save_for_backward(D, weights.detach() if weights is not None else None)
                return D.reshape(z.shape) if z.dim() == 1 else D

            @staticmethod
            @torch.autograd.function.once_differentiable
            def backward(ctx, grad):
                D, w = ctx.saved_tensors
                solver = ctx.solver
                n = D.shape[0]
                k = D.shape[1]
                dev = D.device
                V = _colmajor(grad.reshape(n, -1) if grad.dim() == 1 else grad)
                st = _stream(dev)
                L = _ffi.lib()
                A = torch.empty((k, n), dtype=torch.float64, device=dev).t()
                _ffi.check(L.within_adjoint_rhs(n, k, C.c_void_p(V.data_ptr()),
                                                C.c_void_p(w.data_ptr()) if w is not None else None,
                                                C.c_void_p(A.data_ptr()), st))
                _, S, _ = solver.solve_device(A, ctx.options)
                need_z, need_w = ctx.needs_input_grad[0], ctx.has_w and ctx.needs_input_grad[1]
                gz = torch.empty((k, n), dtype=torch.float64, device=dev).t() if need_z else None
                gw = torch.empty(n, dtype=torch.float64, device=dev) if need_w else None
                if need_z or need_w:
                    _ffi.check(L.within_demean_vjp(
                        n, k, C.c_void_p(D.data_ptr()), C.c_void_p(A.data_ptr()), C.c_void_p(S.data_ptr()),
                        C.c_void_p(w.data_ptr()) if w is not None else None,
                        C.c_void_p(gz.data_ptr()) if gz is not None else None,
                        C.c_void_p(gw.data_ptr()) if gw is not None else None, st))
                if gz is not None:
                    gz = gz.reshape(ctx.shape) if len(ctx.shape) == 1 else gz
                return gz, gw, None, None

        cls._fn = _Demean
        return _Demean


def demean(z, design, weights=None, options=None, preconditioner=None, solver=None):
    """Differentiable ``z - D x*`` for a CUDA float64 tensor ``z`` of shape (n,)
    or (n, k), with gradients with respect to ``z`` and ``weights`` (a CUDA
    float64 tensor of shape (n,), positive).  ``solver`` may be a ``Solver``
    already built for ``design`` and these weights (the forward solve uses the
    solver's weights, the weight gradient the tensor passed here, so the two
    must agree: a solver built with other weights, or with none when weights
    are passed, raises ValueError); otherwise one is built (the
    preconditioner depends on the weights)."""
    from . import Solver
    _check_f64_cuda("z", z)
    if weights is not None:
        _check_f64_cuda("weights", weights)
        if weights.dim() != 1 or weights.shape[0] != z.shape[0]:
            raise ValueError(f"weights must have shape ({z.shape[0]},), got {tuple(weights.shape)}")
        if not bool((weights > 0).all()):
            raise ValueError("weights must be positive for the demeaning gradient")
    if solver is None:
        w_host = None if weights is None else weights.detach().cpu().numpy().astype(np.float64)
        solver = Solver(design, weights=w_host, preconditioner=preconditioner,
                        device=-1 if z.device.index is None else z.device.index)
    if solver.n_obs != z.shape[0]:
        raise ValueError(f"z has {z.shape[0]} rows but the solver has {solver.n_obs} observations")
    fp = getattr(solver, "_weights_fp", None)
    if (weights is None) != (fp is None):
        raise ValueError("the solver was built " + ("with" if fp is not None else "without") +
                         " weights, but demean was called " + ("without" if weights is None else "with") + " them")
    if weights is not None:
        wd = weights.detach()
        got = (float(wd.sum()), float((wd * wd).sum()))
        for a, b in zip(got, fp):
            if abs(a - b) > 1e-10 * max(abs(a), abs(b), 1e-300):
                raise ValueError("the solver was built with other weights than the weights passed to demean")
    return DemeanFunction.get().apply(z, weights, solver, options)
