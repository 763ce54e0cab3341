"""ctypes view of the CPU FP64 restatement (``oracle/build/liboracle.so``).

TEST INFRASTRUCTURE ONLY.  The parity tests, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` use it as the checker; the product package
``within_b200`` never imports it.  See ``within_oracle.h`` for the reference
files each routine restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "liboracle.so")


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class or_precond_cfg(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("exact_local", C.c_int),
        ("ac_seed", C.c_uint64),
        ("ac_split", C.c_uint32),
        ("schur_exact", C.c_int),
        ("schur_seed", C.c_uint64),
        ("schur_split", C.c_uint32),
        ("dense_threshold", C.c_size_t),
        ("scaling_tol", C.c_double),
        ("scaling_max_sweeps", C.c_size_t),
        ("scaling_error", C.c_int),
    ]


class or_stats(C.Structure):
    _fields_ = [
        ("converged", C.c_int),
        ("iterations", C.c_size_t),
        ("residual", C.c_double),
        ("residual_norm", C.c_double),
        ("stop_reason", C.c_int),
        ("time_setup", C.c_double),
        ("time_solve", C.c_double),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        L.or_last_error.restype = C.c_char_p
        L.or_solver_new.argtypes = [C.c_size_t, C.c_size_t, P, P, P, P, C.c_size_t, P, P, P,
                                    C.POINTER(C.c_void_p)]
        L.or_solver_free.argtypes = [P]
        for f in ("or_solver_n_dofs", "or_solver_n_obs", "or_solver_n_terms",
                  "or_solver_n_subdomains", "or_solver_n_warnings"):
            getattr(L, f).argtypes = [P]
            getattr(L, f).restype = C.c_size_t
        L.or_solver_term.argtypes = [P, C.c_size_t, P, P, P, P]
        L.or_solver_obs_perm.argtypes = [P, P]
        L.or_solver_has_precond.argtypes = [P]
        L.or_solver_unidentified.argtypes = [P, P, C.c_size_t]
        L.or_solver_unidentified.restype = C.c_size_t
        L.or_solver_solve.argtypes = [P, P, C.c_double, C.c_size_t, C.c_size_t, P, P, P]
        for f in ("or_solver_apply", "or_solver_apply_adjoint", "or_solver_gather_plain",
                  "or_solver_precond_apply"):
            getattr(L, f).argtypes = [P, P, P]
        L.or_solver_loading.argtypes = [P, C.c_size_t, P]
        L.or_solver_sqrt_weights.argtypes = [P, P]
        L.or_lsmr_dense.argtypes = [C.c_size_t, C.c_size_t, P, P, C.c_double, C.c_size_t,
                                    C.c_size_t, P, P, P]
        L.or_stable_argsort.argtypes = [P, C.c_size_t, C.c_size_t, P]
        L.or_vec_norm.argtypes = [P, C.c_size_t]
        L.or_vec_norm.restype = C.c_double
        L.or_compensated_sum.argtypes = [P, C.c_size_t]
        L.or_compensated_sum.restype = C.c_double
        _lib = L
    return _lib


class OracleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _check(rc: int):
    if rc != 0:
        raise OracleError(rc, lib().or_last_error().decode())


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def precond_cfg(kind: str = "additive", exact_local: bool = False, ac_seed: int = 0,
                ac_split: int = 2, schur_exact: bool = False, schur_seed: int = 0,
                schur_split: int = 1, dense_threshold: int = 24, scaling_tol: float = 1e-9,
                scaling_max_sweeps: int = 2048, scaling_error: bool = False) -> or_precond_cfg:
    k = {"off": 0, "additive": 1, "diagonal": 2}[kind]
    return or_precond_cfg(k, int(exact_local), ac_seed, ac_split, int(schur_exact), schur_seed,
                          schur_split, dense_threshold, scaling_tol, scaling_max_sweeps,
                          int(scaling_error))


@dataclass
class Effect:
    levels: np.ndarray
    intercept: bool = True
    slopes: tuple = ()


def _lower(design):
    """Categories matrix (n, Q) or list of Effect -> flat arrays for the C ABI."""
    if isinstance(design, np.ndarray):
        cats = np.asarray(design, dtype=np.uint32)
        n, q = cats.shape
        codes = np.asfortranarray(cats).ravel(order="F").copy()
        return (n, q, codes, np.ones(q, np.int32), np.zeros(q, np.uintp),
                np.zeros(0, np.uintp), 0, np.zeros(0, np.float64))
    effects = list(design)
    n = len(effects[0].levels)
    codes = np.concatenate([np.asarray(e.levels, np.uint32) for e in effects])
    intercept = np.array([1 if e.intercept else 0 for e in effects], np.int32)
    n_slopes = np.array([len(e.slopes) for e in effects], np.uintp)
    cols = [np.asarray(s, np.float64) for e in effects for s in e.slopes]
    slope_idx = np.arange(len(cols), dtype=np.uintp)
    slopes = np.concatenate(cols) if cols else np.zeros(0, np.float64)
    return n, len(effects), codes, intercept, n_slopes, slope_idx, len(cols), slopes


@dataclass
class OracleResult:
    x: np.ndarray
    demeaned: np.ndarray
    converged: bool
    iterations: int
    residual: float
    residual_norm: float
    stop_reason: int
    time_setup: float
    time_solve: float


class OracleSolver:
    def __init__(self, design, weights=None, cfg: or_precond_cfg | None = None):
        L = lib()
        (self.n_obs, self.n_terms, codes, intercept, n_slopes, slope_idx, nsc,
         slopes) = _lower(design)
        self._keep = (codes, intercept, n_slopes, slope_idx, slopes)
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        h = C.c_void_p()
        rc = L.or_solver_new(self.n_obs, self.n_terms, _ptr(codes), _ptr(intercept),
                             _ptr(n_slopes), _ptr(slope_idx), nsc, _ptr(slopes), _ptr(w),
                             None if cfg is None else C.byref(cfg), C.byref(h))
        _check(rc)
        self._h = h
        self.n_dofs = L.or_solver_n_dofs(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().or_solver_free(h)
            self._h = None

    def term(self, t):
        nl, off, nc, srt = C.c_size_t(), C.c_size_t(), C.c_size_t(), C.c_int()
        lib().or_solver_term(self._h, t, C.byref(nl), C.byref(off), C.byref(nc), C.byref(srt))
        return nl.value, off.value, nc.value, bool(srt.value)

    def obs_perm(self):
        out = np.zeros(self.n_obs, np.uint32)
        return out if lib().or_solver_obs_perm(self._h, _ptr(out)) else None

    @property
    def has_precond(self) -> bool:
        return bool(lib().or_solver_has_precond(self._h))

    @property
    def n_subdomains(self) -> int:
        return lib().or_solver_n_subdomains(self._h)

    @property
    def n_warnings(self) -> int:
        return lib().or_solver_n_warnings(self._h)

    def unidentified(self):
        cap = 4096
        buf = np.zeros(3 * cap, np.uintp)
        k = lib().or_solver_unidentified(self._h, _ptr(buf), cap)
        return [tuple(int(v) for v in buf[3 * i:3 * i + 3]) for i in range(min(k, cap))]

    def solve(self, y, tol=1e-8, maxiter=1000, local_size=0) -> OracleResult:
        y = np.ascontiguousarray(y, np.float64)
        x = np.zeros(self.n_dofs)
        d = np.zeros(self.n_obs)
        st = or_stats()
        _check(lib().or_solver_solve(self._h, _ptr(y), tol, maxiter, local_size or 0, _ptr(x),
                                     _ptr(d), C.byref(st)))
        return OracleResult(x, d, bool(st.converged), int(st.iterations), st.residual,
                            st.residual_norm, st.stop_reason, st.time_setup, st.time_solve)

    def _vec(self, fn, x, n_out):
        x = np.ascontiguousarray(x, np.float64)
        out = np.zeros(n_out)
        _check(getattr(lib(), fn)(self._h, _ptr(x), _ptr(out)))
        return out

    def apply(self, x):
        return self._vec("or_solver_apply", x, self.n_obs)

    def apply_adjoint(self, u):
        return self._vec("or_solver_apply_adjoint", u, self.n_dofs)

    def gather_plain(self, x):
        return self._vec("or_solver_gather_plain", x, self.n_obs)

    def precond_apply(self, r):
        return self._vec("or_solver_precond_apply", r, self.n_dofs)

    def loading(self, k):
        out = np.zeros(self.n_obs)
        _check(lib().or_solver_loading(self._h, k, _ptr(out)))
        return out

    def sqrt_weights(self):
        out = np.zeros(self.n_obs)
        return out if lib().or_solver_sqrt_weights(self._h, _ptr(out)) else None


def stable_argsort(key, n_levels):
    key = np.ascontiguousarray(key, np.uint32)
    perm = np.zeros(len(key), np.uint32)
    lib().or_stable_argsort(_ptr(key), len(key), n_levels, _ptr(perm))
    return perm


def lsmr_dense(a, b, tol=1e-10, maxiter=100, local_size=0, precond_diag=None):
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    r, c = a.shape
    x = np.zeros(c)
    st = or_stats()
    pd = None if precond_diag is None else np.ascontiguousarray(precond_diag, np.float64)
    _check(lib().or_lsmr_dense(r, c, _ptr(a), _ptr(b), tol, maxiter, local_size, _ptr(pd),
                               _ptr(x), C.byref(st)))
    return x, st


def vec_norm(v):
    v = np.ascontiguousarray(v, np.float64)
    return lib().or_vec_norm(_ptr(v), len(v))


def compensated_sum(v):
    v = np.ascontiguousarray(v, np.float64)
    return lib().or_compensated_sum(_ptr(v), len(v))
