"""B200-native fixed-effects projection: the preconditioned modified-LSMR solve
of ``D'WD x = D'W y`` from leostimpfle/within, on sm_100a.

Drop-in for the ``within`` Python API (python/within/__init__.py,
crates/within-py/src/api.rs):

    import numpy as np
    import within_b200 as within

    categories = np.asfortranarray(np.column_stack([a, b]).astype(np.uint32))
    result = within.solve(categories, y)          # SolveResult
    solver = within.Solver(categories)            # reusable preconditioner
    r1, r2 = solver.solve(y1), solver.solve(y2)
    batch = solver.solve_batch(Y)                 # Y: (n_obs, k), one RHS per column

Every solve runs in ``libwithin_gpu.so`` on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import warnings
from dataclasses import dataclass

import numpy as np

from . import _ffi
from . import config
from .config import (AdditiveSchwarz, ApproxCholConfig, ApproxSchurConfig, LocalSolverConfig,
                     ReductionStrategy, ScalingConfig, Schur)

__all__ = [
    "BatchSolveResult",
    "CoefficientLayout",
    "Effect",
    "LsmrOptions",
    "Preconditioner",
    "PreconditionerConfig",
    "SolveResult",
    "Solver",
    "UnidentifiedDirection",
    "solve",
    "solve_batch",
    "demean",
    "SolverSet",
    "solve_many",
    "fwl",
    "FwlResult",
    "default_tuning",
    "Staleness",
    "MlsmrResult",
    "solve_ladder",
    "LadderResult",
    "config",
]


# ---------------------------------------------------------------------------
# configuration objects (crates/within-py/src/config.rs)

class PreconditionerConfig:
    """Preconditioner selection shortcut: ``Additive`` (default), ``Off``, ``Diagonal``."""

    __slots__ = ("kind",)

    def __init__(self, kind: int):
        self.kind = kind

    def __repr__(self) -> str:
        return "PreconditionerConfig." + {0: "Off", 1: "Additive", 2: "Diagonal"}[self.kind]

    def __eq__(self, other):
        return isinstance(other, PreconditionerConfig) and other.kind == self.kind

    def __hash__(self):
        return hash(self.kind)


PreconditionerConfig.Off = PreconditionerConfig(_ffi.PRECOND_OFF)
PreconditionerConfig.Additive = PreconditionerConfig(_ffi.PRECOND_ADDITIVE)
PreconditionerConfig.Diagonal = PreconditionerConfig(_ffi.PRECOND_DIAGONAL)


@dataclass(frozen=True)
class LsmrOptions:
    """LsmrOptions (crates/within/src/config.rs:159-178)."""

    tol: float = 1e-8
    maxiter: int = 1000
    local_size: int | None = None

    def _c(self) -> _ffi.LsmrOptionsC:
        return _ffi.LsmrOptionsC(float(self.tol), int(self.maxiter), int(self.local_size or 0))


@dataclass(frozen=True)
class Staleness:
    """Escalation rule (crates/schwarz-precond/src/lsmr.rs:95-153): hand off
    after ``window`` consecutive iterations whose relative normal-equation
    residual contracted by a ratio above ``threshold`` (in [0, 1))."""

    window: int
    threshold: float

    def __post_init__(self):
        if int(self.window) <= 0:
            raise ValueError("staleness window must be positive")
        if not 0.0 <= float(self.threshold) < 1.0:
            raise ValueError(f"staleness threshold must be in [0, 1), got {self.threshold}")


@dataclass
class MlsmrResult:
    """Device result of :meth:`Solver.mlsmr_device`: X (n_dofs, k) and D
    (n_obs, k) CUDA tensors, per-column convergence and stop reasons
    (LsmrStopReason names, lsmr.rs:54-73)."""

    x: object
    demeaned: object
    converged: list
    iterations: list
    residual: list
    stop_reason: list


class Effect:
    """One term of a design: level codes, an intercept flag, slope covariates
    (crates/within/src/domain/effect.rs:12-42)."""

    __slots__ = ("levels", "intercept", "slopes")

    def __init__(self, levels, intercept: bool = True, slopes=None):
        lv = np.asarray(levels)
        if lv.ndim != 1:
            raise TypeError("levels must be a 1-D uint32 array")
        if lv.dtype != np.uint32:
            if not np.issubdtype(lv.dtype, np.integer):
                raise TypeError(f"levels must be a 1-D uint32 array, got dtype {lv.dtype}")
            if lv.size and lv.min() < 0:
                raise ValueError("levels must be non-negative")
            lv = lv.astype(np.uint32)
        self.levels = np.ascontiguousarray(lv)
        self.intercept = bool(intercept)
        sl = []
        for j, s in enumerate(slopes or []):
            a = np.ascontiguousarray(np.asarray(s, dtype=np.float64))
            if a.ndim != 1:
                raise TypeError(f"slope {j} must be a 1-D float64 array")
            if a.shape[0] != self.levels.shape[0]:
                raise ValueError(f"slope {j} has {a.shape[0]} values, expected {self.levels.shape[0]}")
            sl.append(a)
        self.slopes = tuple(sl)
        if not self.intercept and not self.slopes:
            raise ValueError("an effect must have an intercept or at least one slope")


@dataclass(frozen=True)
class UnidentifiedDirection:
    """A per-level direction the data cannot identify (term, level, column)."""

    term: int
    level: int
    column: int

    def __repr__(self) -> str:
        return f"UnidentifiedDirection(term={self.term}, level={self.level}, column={self.column})"


class CoefficientLayout:
    """Flat ``x`` index <-> (term, level, column) (crates/within/src/solver.rs:125-200)."""

    def __init__(self, terms: list[tuple[int, int, int]], n_dofs: int):
        self._terms = terms  # (offset, n_levels, n_columns)
        self._n_dofs = n_dofs

    def n_dofs(self) -> int:
        return self._n_dofs

    def n_terms(self) -> int:
        return len(self._terms)

    def n_levels(self, term: int) -> int:
        if not 0 <= term < len(self._terms):
            raise IndexError(f"term {term} out of range")
        return self._terms[term][1]

    def n_columns(self, term: int) -> int:
        if not 0 <= term < len(self._terms):
            raise IndexError(f"term {term} out of range")
        return self._terms[term][2]

    def index(self, term: int, level: int, column: int) -> int:
        if not 0 <= term < len(self._terms):
            raise IndexError(f"term {term} out of range")
        off, nl, nc = self._terms[term]
        if not (0 <= level < nl and 0 <= column < nc):
            raise IndexError(f"address ({term}, {level}, {column}) out of range")
        return off + column * nl + level

    def address(self, index: int) -> tuple[int, int, int]:
        if not 0 <= index < self._n_dofs:
            raise IndexError(f"index {index} out of range")
        term = max(t for t, (off, _, _) in enumerate(self._terms) if off <= index)
        off, nl, _ = self._terms[term]
        within = index - off
        return term, within % nl, within // nl


@dataclass
class SolveResult:
    """Result of one solve (crates/within/src/solver.rs:205-242)."""

    x: np.ndarray
    unidentified: list
    layout: CoefficientLayout
    demeaned: np.ndarray
    converged: bool
    iterations: int
    residual: float
    time_total: float
    time_setup: float
    time_solve: float


@dataclass
class BatchSolveResult:
    """Result of a batch solve (solver.rs:246-293); ``x`` is (n_dofs, k), ``demeaned`` (n_obs, k)."""

    x: np.ndarray
    unidentified: list
    layout: CoefficientLayout
    demeaned: np.ndarray
    converged: list
    iterations: list
    residual: list
    time_solve: list
    time_setup: float
    time_total: float


class Preconditioner:
    """Opaque handle to a built preconditioner, reusable across solvers of the
    same design (operator/schwarz.rs:115-183).  It lives on the GPU."""

    def __init__(self, handle):
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _ffi.lib().within_preconditioner_free(h)
            self._h = None

    @property
    def variant_name(self) -> str:
        return _ffi.lib().within_preconditioner_variant_name(self._h).decode()

    def nrows(self) -> int:
        return int(_ffi.lib().within_preconditioner_n(self._h))

    def ncols(self) -> int:
        return self.nrows()

    def stats(self) -> dict:
        """Sizes of the built preconditioner (subdomains, local slots and the
        non-zeros of C, C^T, the factor and the dense blocks)."""
        st = _ffi.PrecondStatsC()
        _ffi.check(_ffi.lib().within_preconditioner_stats(self._h, C.byref(st)))
        return {f: int(getattr(st, f)) for f, _ in _ffi.PrecondStatsC._fields_}

    def apply_device(self, x, y, stream=None) -> None:
        """``y = M^-1 x`` on CUDA float64 tensors of length n (Preconditioner::apply),
        on ``stream`` (a cudaStream_t as int; default torch's current stream, so
        the call is ordered with the torch work that produced ``x``)."""
        _ffi.check(_ffi.lib().within_preconditioner_apply(
            self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), C.c_void_p(_stream_of(x, stream))))

    def __repr__(self) -> str:
        return f"Preconditioner({self.variant_name}, n={self.nrows()})"

    def to_bytes(self) -> bytes:
        """The preconditioner's host image in this library's byte format."""
        L = _ffi.lib()
        n = C.c_uint64()
        _ffi.check(L.within_preconditioner_serialize(self._h, None, 0, C.byref(n)))
        buf = (C.c_uint8 * max(1, n.value))()
        _ffi.check(L.within_preconditioner_serialize(self._h, buf, n.value, C.byref(n)))
        return bytes(buf[:n.value])

    @classmethod
    def from_bytes(cls, data: bytes, device: int = -1) -> "Preconditioner":
        """Uploads a serialised preconditioner to ``device`` (default: current)."""
        data = bytes(data)
        h = C.c_void_p()
        buf = (C.c_uint8 * max(1, len(data))).from_buffer_copy(data or b"\0")
        _ffi.check(_ffi.lib().within_preconditioner_deserialize(buf, len(data), device, C.byref(h)))
        return cls(h)

    def __reduce__(self):
        # pickling (crates/within-py/src/config.rs:366-389): the host image as bytes
        return (Preconditioner.from_bytes, (self.to_bytes(),))


# ---------------------------------------------------------------------------
# lowering helpers

def _precond_config(p) -> _ffi.PrecondConfigC | None:
    """PreconditionerInput resolution (solver.rs:62-110, within-py config.rs)."""
    if p is None:
        return None
    c = _ffi.PrecondConfigC()
    _ffi.lib().within_precond_config_default(C.byref(c))
    if isinstance(p, PreconditionerConfig):
        c.kind = p.kind
        return c
    if isinstance(p, AdditiveSchwarz):
        c.kind = _ffi.PRECOND_ADDITIVE
        ls = p.local_solver or LocalSolverConfig()
        if ls.approx_chol is not None:
            c.approx_chol_seed = ls.approx_chol.seed
            c.approx_chol_split = ls.approx_chol.split_merge or 0
        if ls.schur is not None:
            c.schur_exact = 1 if ls.schur.exact_mode else 0
            if ls.schur.config is not None:
                c.schur_seed = ls.schur.config.seed
                c.schur_split = ls.schur.config.split
        if ls.dense_threshold is not None:
            c.dense_threshold = int(ls.dense_threshold)
        if ls.scaling is not None:
            if ls.scaling.tolerance is not None:
                c.scaling_tolerance = float(ls.scaling.tolerance)
            if ls.scaling.max_sweeps is not None:
                c.scaling_max_sweeps = int(ls.scaling.max_sweeps)
            if ls.scaling.on_failure is not None:
                if ls.scaling.on_failure not in ("warn", "error"):
                    raise ValueError("ScalingConfig.on_failure must be 'warn' or 'error'")
                c.scaling_error = 1 if ls.scaling.on_failure == "error" else 0
        return c
    raise TypeError(f"unsupported preconditioner argument {p!r}")


class _Design:
    def __init__(self, design):
        L = _ffi.lib()
        h = C.c_void_p()
        if isinstance(design, np.ndarray) or hasattr(design, "__array_interface__"):
            cats = np.asarray(design)
            if cats.ndim != 2 or cats.dtype != np.uint32:
                raise TypeError(f"design must be a 2-D uint32 array, got {cats.dtype} with ndim {cats.ndim}")
            if not cats.flags.f_contiguous and cats.shape[1] > 1:
                warnings.warn("categories array is C-ordered; an F-ordered copy is made "
                              "(np.asfortranarray avoids it)", stacklevel=4)
            codes = np.asfortranarray(cats)
            self._keep = codes
            self.n_obs = cats.shape[0]
            _ffi.check(L.within_design_from_categories(_ffi.ptr(codes.reshape(-1, order="F")),
                                                       cats.shape[0], cats.shape[1], C.byref(h)))
        else:
            effects = list(design)
            if not effects or not all(isinstance(e, Effect) for e in effects):
                raise TypeError("design must be a uint32 categories matrix or a list of Effect")
            n = effects[0].levels.shape[0]
            for e in effects:
                if e.levels.shape[0] != n:
                    raise ValueError("all effects must have the same number of observations")
            lv = (C.c_void_p * len(effects))(*[e.levels.ctypes.data for e in effects])
            icpt = np.array([1 if e.intercept else 0 for e in effects], np.int32)
            ns = np.array([len(e.slopes) for e in effects], np.uint64)
            sl_list = [s for e in effects for s in e.slopes]
            sl = (C.c_void_p * max(1, len(sl_list)))(*[s.ctypes.data for s in sl_list])
            self._keep = (effects, lv, icpt, ns, sl)
            self.n_obs = n
            _ffi.check(L.within_design_from_effects(n, len(effects), lv, _ffi.ptr(icpt), _ffi.ptr(ns),
                                                    sl, C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            _ffi.lib().within_design_free(self.h)
            self.h = None


def _stream_of(t, stream):
    """The cudaStream_t to run on: ``stream`` if given, else torch's current
    stream on the tensor's device.  Handle 0 (torch's default stream) becomes
    cudaStreamLegacy: the C ABI reads NULL as "the solver's own stream", which
    is not ordered with torch's work."""
    if stream is None:
        import torch
        stream = torch.cuda.current_stream(t.device).cuda_stream
    return int(stream) or _ffi.CUDA_STREAM_LEGACY


def _as_f64_1d(name, a):
    arr = np.asarray(a)
    if arr.ndim != 1 or arr.dtype != np.float64:
        raise TypeError(f"{name} must be a 1-D float64 array, got dtype {arr.dtype}")
    return np.ascontiguousarray(arr)


def _out_f64_1d(name, a, n):
    if not isinstance(a, np.ndarray) or a.ndim != 1 or a.dtype != np.float64 or not a.flags.c_contiguous \
            or not a.flags.writeable:
        raise TypeError(f"{name} must be a writeable contiguous 1-D float64 array")
    if a.shape[0] != n:
        raise ValueError(f"{name} has length {a.shape[0]}, expected {n}")
    return a


def _as_f64_2d(name, a):
    arr = np.asarray(a)
    if arr.ndim != 2 or arr.dtype != np.float64:
        raise TypeError(f"{name} must be a 2-D float64 array, got dtype {arr.dtype}")
    return np.asfortranarray(arr)


# ---------------------------------------------------------------------------

def default_tuning() -> dict:
    """The default within_tuning record (within_tuning_default) as a dict."""
    t = _ffi.TuningC()
    _ffi.lib().within_tuning_default(C.byref(t))
    return {f: getattr(t, f) for f, _ in _ffi.TuningC._fields_}


def _tuning_struct(tuning, design, weights):
    """The within_tuning record of a Solver: None (the defaults and the WITHIN_*
    environment overrides), "auto" (the autotuner's table entry nearest to the
    design, else None), or a dict of within_tuning fields over the defaults."""
    if tuning is None:
        return None
    if isinstance(tuning, str):
        if tuning != "auto":
            raise ValueError(f"tuning must be None, 'auto' or a dict, got {tuning!r}")
        from . import autotune
        table = autotune.load_table()
        if not table:
            return None
        if isinstance(design, np.ndarray) or hasattr(design, "__array_interface__"):
            cats = np.asarray(design)
            levels = [int(cats[:, t].max()) + 1 if cats.shape[0] else 0 for t in range(cats.shape[1])]
            n, slopes = cats.shape[0], False
        else:
            effects = list(design)
            levels = [int(e.levels.max()) + 1 if e.levels.size else 0 for e in effects]
            n, slopes = effects[0].levels.shape[0], any(e.slopes for e in effects)
        rec = autotune.lookup(autotune.design_key(n, levels, slopes, weights is not None), table)
        if rec is None:
            return None
        tuning = rec
    t = _ffi.TuningC()
    _ffi.lib().within_tuning_default(C.byref(t))
    for k, v in dict(tuning).items():
        if k not in dict(_ffi.TuningC._fields_):
            raise ValueError(f"unknown tuning field {k!r}")
        setattr(t, k, v)
    return t


class Solver:
    """Persistent solver owning its preconditioner (crates/within/src/solver.rs:295-593).

    ``tuning``: "auto" (default) takes the kernel variants and factor stop
    rules of the autotuner's table entry nearest to the design
    (within_b200/autotune.py), None the built-in defaults (with the WITHIN_*
    environment overrides), or a dict of within_tuning fields."""

    def __init__(self, design, weights=None, preconditioner=None, device: int = -1,
                 precision: str = "fp64", tuning="auto"):
        L = _ffi.lib()
        d = _Design(design)
        w = None if weights is None else _as_f64_1d("weights", weights)
        if w is not None and w.shape[0] != d.n_obs:
            raise ValueError(f"weights has length {w.shape[0]}, expected {d.n_obs}")
        # fingerprint of the weights (sum and sum of squares), which demean()
        # checks a caller's weights tensor against when given this solver
        self._weights_fp = None if w is None else (float(np.sum(w)), float(np.sum(w * w)))
        prebuilt = preconditioner._h if isinstance(preconditioner, Preconditioner) else None
        cfg = None if prebuilt is not None else _precond_config(preconditioner)
        tn = _tuning_struct(tuning, design, w)
        self.tuning = None if tn is None else {f: getattr(tn, f) for f, _ in _ffi.TuningC._fields_}
        h = C.c_void_p()
        if tn is None:
            _ffi.check(L.within_solver_new(d.h, _ffi.ptr(w), None if cfg is None else C.byref(cfg),
                                           prebuilt, device, C.byref(h)))
        else:
            _ffi.check(L.within_solver_new_tuned(d.h, _ffi.ptr(w), None if cfg is None else C.byref(cfg),
                                                 prebuilt, device, C.byref(tn), C.byref(h)))
        self._h = h
        self._n_obs = int(L.within_solver_n_obs(h))
        self._n_dofs = int(L.within_solver_n_dofs(h))
        terms = []
        for t in range(int(L.within_solver_n_terms(h))):
            nl, off, nc = C.c_uint64(), C.c_uint64(), C.c_uint64()
            _ffi.check(L.within_solver_term_layout(h, t, C.byref(nl), C.byref(off), C.byref(nc)))
            terms.append((off.value, nl.value, nc.value))
        self._layout = CoefficientLayout(terms, self._n_dofs)
        self._precision = "fp64"
        self.set_precision(precision)
        cap = 1 << 16
        buf = np.zeros(3 * cap, np.uint64)
        k = int(L.within_solver_unidentified(h, _ffi.ptr(buf), cap))
        self._unidentified = [UnidentifiedDirection(int(buf[3 * i]), int(buf[3 * i + 1]), int(buf[3 * i + 2]))
                              for i in range(min(k, cap))]
        nw = int(L.within_solver_n_warnings(h))
        for _ in range(nw):
            warnings.warn("signed component: dominance scaling uncertified; deficits clamped, "
                          "preconditioner quality may degrade", UserWarning, stacklevel=2)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _ffi.lib().within_solver_free(h)
            self._h = None

    @property
    def n_dofs(self) -> int:
        return self._n_dofs

    @property
    def precision(self) -> str:
        return self._precision

    def set_precision(self, precision: str) -> None:
        """"fp64" (default, the reference's arithmetic) or "mixed": FP64
        iterative refinement on the normal-equation residual around an inner
        solve whose vectors, operator data and factors are stored in FP32."""
        code = {"fp64": _ffi.PRECISION_FP64, "mixed": _ffi.PRECISION_MIXED}.get(precision)
        if code is None:
            raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")
        _ffi.check(_ffi.lib().within_solver_set_precision(self._h, code))
        self._precision = precision

    @property
    def n_obs(self) -> int:
        return self._n_obs

    @property
    def layout(self) -> CoefficientLayout:
        return self._layout

    @property
    def preconditioner(self) -> Preconditioner | None:
        h = _ffi.lib().within_solver_preconditioner(self._h)
        return Preconditioner(C.c_void_p(h)) if h else None

    @property
    def handle(self):
        return self._h

    def obs_perm(self) -> np.ndarray | None:
        out = np.zeros(self._n_obs, np.uint32)
        return out if _ffi.lib().within_solver_obs_perm(self._h, _ffi.ptr(out)) else None

    def solve(self, y, options: LsmrOptions | None = None, *, x_out=None, demeaned_out=None) -> SolveResult:
        """Solver::solve (solver.rs:503-527).  ``x_out`` / ``demeaned_out``
        (optional, 1-D float64 of n_dofs / n_obs) receive the results in
        place; page-locked buffers (e.g. ``torch.empty(n, dtype=torch.float64,
        pin_memory=True).numpy()``), like a page-locked ``y``, are copied by
        DMA directly, pageable ones through the library's staging slots."""
        y = _as_f64_1d("y", y)
        if y.shape[0] != self._n_obs:
            raise ValueError(f"response vector length ({y.shape[0]}) does not match number of "
                             f"observations ({self._n_obs})")
        x = np.zeros(self._n_dofs) if x_out is None else _out_f64_1d("x_out", x_out, self._n_dofs)
        dm = np.zeros(self._n_obs) if demeaned_out is None else _out_f64_1d("demeaned_out", demeaned_out,
                                                                             self._n_obs)
        st = _ffi.SolveStatsC()
        opts = (options or LsmrOptions())._c()
        _ffi.check(_ffi.lib().within_solver_solve(self._h, _ffi.ptr(y), C.byref(opts), _ffi.ptr(x),
                                                  _ffi.ptr(dm), C.byref(st)))
        return SolveResult(x, list(self._unidentified), self._layout, dm, bool(st.converged),
                           int(st.iterations), float(st.residual), st.time_total, st.time_setup,
                           st.time_solve)

    def solve_batch(self, Y, options: LsmrOptions | None = None) -> BatchSolveResult:
        Y = _as_f64_2d("Y", Y)
        if Y.shape[0] != self._n_obs:
            raise ValueError(f"Y has {Y.shape[0]} rows but solver has {self._n_obs} observations")
        k = Y.shape[1]
        X = np.zeros((self._n_dofs, k), order="F")
        D = np.zeros((self._n_obs, k), order="F")
        st = (_ffi.SolveStatsC * max(1, k))()
        opts = (options or LsmrOptions())._c()
        if k:
            _ffi.check(_ffi.lib().within_solver_solve_batch(self._h, _ffi.ptr(Y), k, C.byref(opts),
                                                            _ffi.ptr(X), _ffi.ptr(D), st))
        return BatchSolveResult(X, list(self._unidentified), self._layout, D,
                                [bool(st[i].converged) for i in range(k)],
                                [int(st[i].iterations) for i in range(k)],
                                [float(st[i].residual) for i in range(k)],
                                [st[i].time_solve for i in range(k)], 0.0,
                                max([st[i].time_total for i in range(k)] or [0.0]))

    def solve_device(self, Y, options: LsmrOptions | None = None, X=None, D=None, stream=None):
        """Device-resident solve_batch on CUDA float64 tensors (column-major (n_obs, k)
        storage: pass ``Y.t().contiguous().t()`` or a 1-D tensor for k = 1)."""
        import torch
        if Y.dtype != torch.float64 or not Y.is_cuda:
            raise TypeError("Y must be a CUDA float64 tensor")
        k = 1 if Y.dim() == 1 else Y.shape[1]
        if X is None:
            X = torch.empty((k, self._n_dofs), dtype=torch.float64, device=Y.device).t()
        if D is None:
            D = torch.empty((k, self._n_obs), dtype=torch.float64, device=Y.device).t()
        st = (_ffi.SolveStatsC * k)()
        opts = (options or LsmrOptions())._c()
        _ffi.check(_ffi.lib().within_solver_solve_batch_device(
            self._h, C.c_void_p(Y.data_ptr()), k, C.byref(opts), C.c_void_p(X.data_ptr()),
            C.c_void_p(D.data_ptr()), st, C.c_void_p(_stream_of(Y, stream))))
        stats = [(bool(st[i].converged), int(st[i].iterations), float(st[i].residual)) for i in range(k)]
        return X, D, stats

    def mlsmr_device(self, Y, options: LsmrOptions | None = None, warm_start=None,
                     escalation: Staleness | None = None, X=None, D=None, stream=None) -> MlsmrResult:
        """solve_device with the MlsmrOptions extras (lsmr.rs:155-171):
        ``warm_start`` a CUDA float64 (n_dofs,) or (n_dofs, k) tensor in x's
        layout (column-major storage for k > 1), ``escalation`` a Staleness
        rule.  Designs with slope terms take no warm start."""
        import torch
        if Y.dtype != torch.float64 or not Y.is_cuda:
            raise TypeError("Y must be a CUDA float64 tensor")
        k = 1 if Y.dim() == 1 else Y.shape[1]
        if X is None:
            X = torch.empty((k, self._n_dofs), dtype=torch.float64, device=Y.device).t()
        if D is None:
            D = torch.empty((k, self._n_obs), dtype=torch.float64, device=Y.device).t()
        ext = _ffi.SolveExtC(None, 0, 0.0)
        if warm_start is not None:
            x0 = warm_start
            if x0.dtype != torch.float64 or not x0.is_cuda:
                raise TypeError("warm_start must be a CUDA float64 tensor")
            if (x0.dim() == 1 and (k != 1 or x0.shape[0] != self._n_dofs)) or \
                    (x0.dim() == 2 and tuple(x0.shape) != (self._n_dofs, k)):
                raise ValueError(f"warm-start shape {tuple(x0.shape)} does not match ({self._n_dofs}, {k})")
            if x0.dim() == 2 and not (x0.stride(0) == 1 and x0.stride(1) == self._n_dofs):
                x0 = x0.t().contiguous().t()
            ext.x0_dev = x0.data_ptr()
        if escalation is not None:
            ext.stale_window = int(escalation.window)
            ext.stale_threshold = float(escalation.threshold)
        st = (_ffi.SolveStatsC * k)()
        stops = (C.c_int32 * k)()
        opts = (options or LsmrOptions())._c()
        _ffi.check(_ffi.lib().within_solver_solve_batch_device_ext(
            self._h, C.c_void_p(Y.data_ptr()), k, C.byref(opts), C.byref(ext), C.c_void_p(X.data_ptr()),
            C.c_void_p(D.data_ptr()), st, stops, C.c_void_p(_stream_of(Y, stream))))
        return MlsmrResult(X, D, [bool(st[i].converged) for i in range(k)], [int(st[i].iterations) for i in range(k)],
                           [float(st[i].residual) for i in range(k)],
                           [_ffi.STOP_REASONS[stops[i]] if 0 <= stops[i] < len(_ffi.STOP_REASONS) else "None"
                            for i in range(k)])

    # Operator trait plumbing (internal observation order, device buffers), on
    # ``stream`` (default torch's current stream: ordered with the torch work
    # around the call, and asynchronous like any torch op)
    def operator_apply_device(self, x, y, stream=None) -> None:
        _ffi.check(_ffi.lib().within_solver_operator_apply(
            self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), C.c_void_p(_stream_of(x, stream))))

    def operator_apply_adjoint_device(self, u, y, stream=None) -> None:
        _ffi.check(_ffi.lib().within_solver_operator_apply_adjoint(
            self._h, C.c_void_p(u.data_ptr()), C.c_void_p(y.data_ptr()), C.c_void_p(_stream_of(u, stream))))


def solve(design, y, weights=None, options: LsmrOptions | None = None, preconditioner=None) -> SolveResult:
    """One-shot ``Solver(design, weights, preconditioner).solve(y, options)``
    (crates/within/src/solver.rs:611-626)."""
    import time
    t0 = time.perf_counter()
    s = Solver(design, weights, preconditioner)
    t1 = time.perf_counter()
    r = s.solve(y, options)
    r.time_setup += t1 - t0
    r.time_total = time.perf_counter() - t0
    return r


def solve_batch(design, Y, weights=None, options: LsmrOptions | None = None,
                preconditioner=None) -> BatchSolveResult:
    """One-shot batch solve (solver.rs:632-646)."""
    import time
    t0 = time.perf_counter()
    s = Solver(design, weights, preconditioner)
    t1 = time.perf_counter()
    Ya = np.asarray(Y)
    if Ya.ndim == 2 and Ya.shape[0] != s.n_obs:
        raise ValueError(f"Y has {Ya.shape[0]} rows but the design has {s.n_obs} observations")
    r = s.solve_batch(Y, options)
    r.time_setup = t1 - t0
    r.time_total = time.perf_counter() - t0
    return r


class SolverSet:
    """Many independent designs solved together (no counterpart in the
    reference, which has one design per ``Solver``): ``within_solvers_new``
    builds one solver per design with the set-up spread over host threads, and
    ``solve_batch`` solves every design's right-hand sides with ``threads``
    host threads driving the designs' streams concurrently on the GPU.  Each
    design keeps its own LSMR state and per-column convergence."""

    def __init__(self, designs, weights=None, preconditioner=None, device: int = -1, threads: int = 8,
                 precision: str = "fp64"):
        L = _ffi.lib()
        self._designs = [_Design(d) for d in designs]
        n = len(self._designs)
        ws = [None] * n if weights is None else [None if w is None else _as_f64_1d("weights", w)
                                                  for w in weights]
        if len(ws) != n:
            raise ValueError(f"{len(ws)} weight vectors for {n} designs")
        for i, (d, w) in enumerate(zip(self._designs, ws)):
            if w is not None and w.shape[0] != d.n_obs:
                raise ValueError(f"weights {i} has length {w.shape[0]}, expected {d.n_obs}")
        dh = (C.c_void_p * max(1, n))(*[d.h.value for d in self._designs])
        wh = (C.c_void_p * max(1, n))(*[None if w is None else w.ctypes.data for w in ws])
        cfg = _precond_config(preconditioner)
        out = (C.c_void_p * max(1, n))()
        self._threads = int(threads)
        _ffi.check(L.within_solvers_new(n, dh, wh, None if cfg is None else C.byref(cfg), device,
                                        self._threads, out))
        self._h = [C.c_void_p(out[i]) for i in range(n)]
        self._n_obs = [int(L.within_solver_n_obs(h)) for h in self._h]
        self._n_dofs = [int(L.within_solver_n_dofs(h)) for h in self._h]
        for h in self._h:
            _ffi.check(L.within_solver_set_precision(
                h, {"fp64": _ffi.PRECISION_FP64, "mixed": _ffi.PRECISION_MIXED}[precision]))

    def __len__(self) -> int:
        return len(self._h)

    def set_precision(self, precision: str) -> None:
        """Solver.set_precision on every design of the set."""
        code = {"fp64": _ffi.PRECISION_FP64, "mixed": _ffi.PRECISION_MIXED}.get(precision)
        if code is None:
            raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")
        for h in self._h:
            _ffi.check(_ffi.lib().within_solver_set_precision(h, code))

    def __del__(self):
        for h in getattr(self, "_h", []):
            if h:
                _ffi.lib().within_solver_free(h)
        self._h = []

    @property
    def n_obs(self) -> list[int]:
        return list(self._n_obs)

    @property
    def n_dofs(self) -> list[int]:
        return list(self._n_dofs)

    def solve_batch(self, Ys, options: LsmrOptions | None = None, want_x: bool = True):
        """``Ys[i]``: (n_obs_i, k_i) float64 (or 1-D).  Returns one
        (x, demeaned, converged, iterations) tuple per design."""
        n = len(self._h)
        if len(Ys) != n:
            raise ValueError(f"{len(Ys)} right-hand-side blocks for {n} designs")
        Yf = []
        for i, Y in enumerate(Ys):
            Y = np.asarray(Y)
            Y = Y.reshape(-1, 1) if Y.ndim == 1 else Y
            Y = _as_f64_2d("Y", Y)
            if Y.shape[0] != self._n_obs[i]:
                raise ValueError(f"Y[{i}] has {Y.shape[0]} rows, design has {self._n_obs[i]}")
            Yf.append(Y)
        ks = np.array([Y.shape[1] for Y in Yf], np.uint64)
        X = [np.zeros((self._n_dofs[i], Yf[i].shape[1]), order="F") for i in range(n)] if want_x else None
        D = [np.zeros(Y.shape, order="F") for Y in Yf]
        st = [(_ffi.SolveStatsC * max(1, int(k)))() for k in ks]
        yp = (C.c_void_p * max(1, n))(*[Y.ctypes.data for Y in Yf])
        xp = (C.c_void_p * max(1, n))(*[x.ctypes.data for x in X]) if want_x else None
        dp = (C.c_void_p * max(1, n))(*[d.ctypes.data for d in D])
        sp = (C.c_void_p * max(1, n))(*[C.addressof(x) for x in st])
        hp = (C.c_void_p * max(1, n))(*[h.value for h in self._h])
        opts = (options or LsmrOptions())._c()
        _ffi.check(_ffi.lib().within_solvers_solve_batch(n, hp, yp, _ffi.ptr(ks), C.byref(opts), xp, dp, sp,
                                                         self._threads))
        return [((X[i] if want_x else None), D[i], [bool(st[i][j].converged) for j in range(int(ks[i]))],
                 [int(st[i][j].iterations) for j in range(int(ks[i]))]) for i in range(n)]


def solve_many(designs, Ys, weights=None, options: LsmrOptions | None = None, preconditioner=None,
               threads: int = 8, precision: str = "fp64"):
    """One-shot ``SolverSet(designs, weights, preconditioner).solve_batch(Ys)``."""
    return SolverSet(designs, weights, preconditioner, threads=threads, precision=precision).solve_batch(Ys, options)


@dataclass
class LadderResult:
    """Result of :func:`solve_ladder`: x / demeaned (host, (n_dofs, k) and
    (n_obs, k)), per column the rung that finished it, its convergence, the
    iterations of every rung summed, and the stop reason of the last rung."""

    x: np.ndarray
    demeaned: np.ndarray
    rung: list
    converged: list
    iterations: list
    stop_reason: list


def solve_ladder(design, Y, weights=None, options: LsmrOptions | None = None,
                 escalation: Staleness = Staleness(4, 0.7), device: int = -1) -> LadderResult:
    """A two-rung preconditioner ladder (warm starts and escalation,
    crates/schwarz-precond/src/lsmr.rs:83-171, the pattern of its
    test_mlsmr_ladder_warm_starts_and_escalates): every column is solved with
    the diagonal preconditioner under the staleness rule; the columns that
    escalate continue on the additive Schwarz preconditioner (built only if
    needed), warm-started from the diagonal rung's iterate.  Both rungs run on
    the GPU; the tolerance stays relative to each column's original ||b||."""
    import torch
    Ya = np.asarray(Y, dtype=np.float64)
    Ya = Ya.reshape(-1, 1) if Ya.ndim == 1 else Ya
    opts = options or LsmrOptions()
    dev = torch.device("cuda", torch.cuda.current_device() if device < 0 else device)
    weak = Solver(design, weights, PreconditionerConfig.Diagonal, device=dev.index)
    Yd = torch.from_numpy(np.ascontiguousarray(Ya.T)).to(dev).t()
    r1 = weak.mlsmr_device(Yd, opts, escalation=escalation)
    X = r1.x.clone()
    D = r1.demeaned.clone()
    k = Ya.shape[1]
    rung = ["Diagonal"] * k
    conv, its, stops = list(r1.converged), list(r1.iterations), list(r1.stop_reason)
    esc = [j for j in range(k) if r1.stop_reason[j] == "Escalated"]
    if esc:
        strong = Solver(design, weights, None, device=dev.index)
        Ye = Yd[:, esc].t().contiguous().t()
        X0 = r1.x[:, esc].t().contiguous().t()
        r2 = strong.mlsmr_device(Ye, opts, warm_start=X0)
        for i, j in enumerate(esc):
            X[:, j] = r2.x[:, i]
            D[:, j] = r2.demeaned[:, i]
            rung[j] = "Additive"
            conv[j] = r2.converged[i]
            its[j] += r2.iterations[i]
            stops[j] = r2.stop_reason[i]
    return LadderResult(X.cpu().numpy(), D.cpu().numpy(), rung, conv, its, stops)


@dataclass
class FwlResult:
    """Frisch-Waugh-Lovell regression of y on X absorbing the fixed effects:
    ``beta`` (p,), the demeaned response and covariates, and the solve's
    per-column convergence."""

    beta: np.ndarray
    demeaned_y: np.ndarray
    demeaned_X: np.ndarray
    converged: list
    iterations: list


def fwl(design, y, X, weights=None, options: LsmrOptions | None = None, preconditioner=None,
        solver: "Solver | None" = None, device: int = -1) -> FwlResult:
    """The FWL regression step after solve_batch (README.md:54-65 of the
    reference): demean [y, X] in one multi-RHS solve on the GPU, then solve the
    least-squares problem min ||W^{1/2} (y~ - X~ beta)|| on the GPU by a QR
    factorisation of the weighted demeaned covariates (FP64), so the n x p
    columns never leave the device.  ``solver`` reuses a built Solver of the
    same design and weights."""
    import torch
    y = _as_f64_1d("y", y)
    Xa = np.asarray(X, dtype=np.float64)
    if Xa.ndim == 1:
        Xa = Xa.reshape(-1, 1)
    if Xa.shape[0] != y.shape[0]:
        raise ValueError(f"X has {Xa.shape[0]} rows, y has {y.shape[0]}")
    s = solver if solver is not None else Solver(design, weights, preconditioner, device=device)
    if s.n_obs != y.shape[0]:
        raise ValueError(f"y has {y.shape[0]} rows but the solver has {s.n_obs} observations")
    dev = torch.device("cuda", torch.cuda.current_device() if device < 0 else device)
    p = Xa.shape[1]
    Y = torch.empty((p + 1, s.n_obs), dtype=torch.float64, device=dev)
    Y[0].copy_(torch.from_numpy(y))
    Y[1:].copy_(torch.from_numpy(np.ascontiguousarray(Xa.T)))
    _, D, stats = s.solve_device(Y.t(), options)
    yt, Xt = D[:, 0], D[:, 1:]
    if weights is not None:
        sw = torch.from_numpy(np.sqrt(_as_f64_1d("weights", weights))).to(dev)
        yw, Xw = yt * sw, Xt * sw[:, None]
    else:
        yw, Xw = yt, Xt
    Qm, Rm = torch.linalg.qr(Xw, mode="reduced")
    beta = torch.linalg.solve_triangular(Rm, (Qm.t() @ yw).unsqueeze(1), upper=True).squeeze(1)
    return FwlResult(beta.cpu().numpy(), yt.cpu().numpy(), Xt.cpu().numpy(),
                     [c for c, _, _ in stats], [it for _, it, _ in stats])


from .autograd import demean  # noqa: E402  (differentiable demeaning; imports torch lazily)
