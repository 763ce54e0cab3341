"""ctypes binding of ``libwithin_gpu.so`` (declared in ``include/within_gpu.h``).

The library is required: importing this module without it raises, and every
solve runs on the GPU through it.  There is no CPU code path.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libwithin_gpu.so")

WITHIN_OK = 0
ERR_INVALID_INPUT = 1
ERR_BUILD = 2
ERR_UNSCALABLE = 3
ERR_SINGULAR = 4
ERR_INDEFINITE = 5
ERR_DIMENSION = 6
ERR_CUDA = 7
ERR_UNSUPPORTED = 8

PRECOND_OFF = 0
PRECOND_ADDITIVE = 1
PRECOND_DIAGONAL = 2

PRECISION_FP64 = 0
PRECISION_MIXED = 1
# cudaStreamLegacy: the legacy default stream (torch's default stream) as a
# non-NULL handle, so a call on it is ordered with torch's work
CUDA_STREAM_LEGACY = 1


class PrecondConfigC(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("approx_chol_seed", C.c_uint64),
        ("approx_chol_split", C.c_uint32),
        ("schur_exact", C.c_int32),
        ("schur_seed", C.c_uint64),
        ("schur_split", C.c_uint32),
        ("dense_threshold", C.c_uint64),
        ("scaling_tolerance", C.c_double),
        ("scaling_max_sweeps", C.c_uint64),
        ("scaling_error", C.c_int32),
        ("reduction", C.c_int32),
    ]


class LsmrOptionsC(C.Structure):
    _fields_ = [("tol", C.c_double), ("maxiter", C.c_uint64), ("local_size", C.c_uint64)]


class SolveStatsC(C.Structure):
    _fields_ = [
        ("converged", C.c_int32),
        ("iterations", C.c_uint64),
        ("residual", C.c_double),
        ("time_total", C.c_double),
        ("time_setup", C.c_double),
        ("time_solve", C.c_double),
    ]


class SolveExtC(C.Structure):
    _fields_ = [("x0_dev", C.c_void_p), ("stale_window", C.c_uint64), ("stale_threshold", C.c_double)]


STOP_REASONS = ["ZeroRhs", "InitialNormalEquationResidualZero", "ResidualTolerance", "NormalEquationTolerance",
                "WarmStartExact", "MaxIterations", "Escalated"]


class TuningC(C.Structure):
    _fields_ = [("staged_sweep", C.c_int32), ("wide_mean_len", C.c_uint32), ("fuse_rounds", C.c_int32),
                ("thread_per_segment", C.c_int32), ("core_dense_max", C.c_uint32), ("core_min_frac", C.c_double),
                ("max_rounds", C.c_uint32), ("core_small", C.c_uint32), ("core_dense_late", C.c_uint32),
                ("warp_ranges", C.c_int32), ("gpu_cross_tab", C.c_int32),
                ("vector_rows", C.c_int32)]


class PrecondStatsC(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in ("n", "n_subdomains", "n_slots", "nnz_c", "nnz_ct", "nnz_fwd",
                                          "nnz_bwd", "nnz_dense", "nnz_core", "n_reduced", "n_rounds")]


# (name, restype, argtypes) of every exported entry point in within_gpu.h
P = C.c_void_p
U64 = C.c_uint64
_SIGNATURES = [
    ("within_precond_config_default", None, [C.POINTER(PrecondConfigC)]),
    ("within_lsmr_options_default", None, [C.POINTER(LsmrOptionsC)]),
    ("within_design_from_categories", C.c_int, [P, U64, U64, C.POINTER(P)]),
    ("within_design_from_effects", C.c_int, [U64, U64, P, P, P, P, C.POINTER(P)]),
    ("within_design_free", None, [P]),
    ("within_design_n_obs", U64, [P]),
    ("within_design_n_dofs", U64, [P]),
    ("within_solver_new", C.c_int, [P, P, P, P, C.c_int32, C.POINTER(P)]),
    ("within_solver_free", None, [P]),
    ("within_solver_n_obs", U64, [P]),
    ("within_solver_n_dofs", U64, [P]),
    ("within_solver_n_warnings", U64, [P]),
    ("within_solver_unidentified", U64, [P, P, U64]),
    ("within_solver_n_terms", U64, [P]),
    ("within_solver_term_layout", C.c_int, [P, U64, P, P, P]),
    ("within_solver_obs_perm", C.c_int, [P, P]),
    ("within_solver_preconditioner", P, [P]),
    ("within_solver_set_precision", C.c_int, [P, C.c_int32]),
    ("within_solver_solve", C.c_int, [P, P, P, P, P, P]),
    ("within_solver_solve_batch", C.c_int, [P, P, U64, P, P, P, P]),
    ("within_solver_solve_batch_device", C.c_int, [P, P, U64, P, P, P, P, P]),
    ("within_solve", C.c_int, [P, P, P, P, P, P, P, P]),
    ("within_solve_batch", C.c_int, [P, P, U64, P, P, P, P, P, P]),
    ("within_solver_operator_apply", C.c_int, [P, P, P, P]),
    ("within_solver_operator_apply_adjoint", C.c_int, [P, P, P, P]),
    ("within_solver_operator_apply_adjoint_noalloc", C.c_int, [P, P, P, P]),
    ("within_solvers_new", C.c_int, [U64, P, P, P, C.c_int32, C.c_uint32, P]),
    ("within_solvers_solve_batch", C.c_int, [U64, P, P, P, P, P, P, P, C.c_uint32]),
    ("within_preconditioner_free", None, [P]),
    ("within_preconditioner_n", U64, [P]),
    ("within_preconditioner_variant_name", C.c_char_p, [P]),
    ("within_preconditioner_stats", C.c_int, [P, P]),
    ("within_tuning_default", None, [P]),
    ("within_solver_new_tuned", C.c_int, [P, P, P, P, C.c_int32, P, P]),
    ("within_solver_solve_batch_device_ext", C.c_int, [P, P, U64, P, P, P, P, P, P, P]),
    ("within_preconditioner_serialize", C.c_int, [P, P, U64, P]),
    ("within_preconditioner_deserialize", C.c_int, [P, U64, C.c_int32, P]),
    ("within_preconditioner_apply", C.c_int, [P, P, P, P]),
    ("within_adjoint_rhs", C.c_int, [U64, U64, P, P, P, P]),
    ("within_demean_vjp", C.c_int, [U64, U64, P, P, P, P, P, P, P]),
    ("within_last_error", C.c_char_p, []),
    ("within_launch_count", U64, []),
    ("within_launch_count_reset", None, []),
]

_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"within_b200: CUDA library {LIB_PATH} is missing; build it with "
                "`python -m within_b200._build` (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, res, args in _SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return [s[0] for s in _SIGNATURES]


class WithinError(RuntimeError):
    """Raised for device or runtime failures (SolveError beyond invalid input)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class WithinValueError(ValueError):
    """Raised for invalid inputs and build errors (BuildError / InvalidInput)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def check(rc: int) -> None:
    if rc == WITHIN_OK:
        return
    msg = lib().within_last_error().decode(errors="replace")
    # Input validation maps to ValueError, runtime failures to RuntimeError
    # (crates/within-py/src/convert.rs:17-42).
    if rc in (ERR_INVALID_INPUT, ERR_BUILD, ERR_UNSCALABLE, ERR_SINGULAR, ERR_DIMENSION):
        raise WithinValueError(rc, msg)
    raise WithinError(rc, msg)


def ptr(a) -> C.c_void_p | None:
    if a is None:
        return None
    return C.c_void_p(a.ctypes.data)
