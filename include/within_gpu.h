/*
 * within_gpu.h -- C ABI of the B200 (sm_100a) fixed-effects solve library
 * `libwithin_gpu.so`.
 *
 * It is a drop-in for leostimpfle/within's preconditioned modified-LSMR solve
 * of D'WD x = D'W y.  Every entry point names the reference interface it
 * replaces (paths relative to the reference checkout).  Plain pointers and
 * sizes only; no torch or CUDA runtime types cross the boundary (streams are
 * passed as `void*` holding a cudaStream_t, NULL = the library's own stream).
 *
 * Conventions
 *  - Return value: WITHIN_OK (0) or one of the WITHIN_ERR_* codes; the message
 *    of the last failure on the calling thread is within_last_error().
 *  - "host" buffers are ordinary CPU memory (pageable or pinned); "dev" buffers
 *    are device pointers on the solver's device.
 *  - Observation vectors are in the caller's order unless a name says
 *    "internal" (the design's locality-sorted order, domain.rs:225-238).
 *  - Multi-RHS arrays are column-major: column j of Y (n_obs x k) starts at
 *    Y + j*n_obs, as in BatchSolveResult (solver.rs:246-293).
 *  - Non-convergence is not an error: stats.converged = 0 (lsmr.rs:363-370).
 *  - Streams: NULL selects the solver's own (non-blocking) stream and the call
 *    returns after its work is done; any other handle (cudaStreamLegacy = 1
 *    for the legacy default stream included) orders the call after the work
 *    already queued there, and the operator applies return without waiting.
 *    Solves and within_preconditioner_apply always wait for their result.
 *  - Threads: every entry point may be called from any thread.  Calls on one
 *    within_solver (solve, solve_batch, the operator applies, set_precision)
 *    take that solver's mutex, so concurrent calls on one handle are safe and
 *    run one after another: a second caller waits for the whole of the first
 *    call (for a solve, its set-up, LSMR loop and result copies).  That
 *    mirrors the reference's Solver::solve(&self) (solver.rs:503-527, shared
 *    across threads in tests/test_free_threaded.py:32-58) without a per-call
 *    workspace pool: a workspace is sized for the whole design (for the 10M-
 *    row panel ~0.7 GB per column bucket), so one per caller would multiply
 *    the memory.  For device overlap, give each thread its own solver, or use
 *    within_solvers_solve_batch.  A preconditioner handle shared by several
 *    solvers is read-only during solves; its per-solver plans live in each
 *    solver.
 */
#ifndef WITHIN_GPU_H
#define WITHIN_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes: crates/within/src/error.rs:9-146 and
 * crates/schwarz-precond/src/error.rs:63-90. */
#define WITHIN_OK 0
#define WITHIN_ERR_INVALID_INPUT 1   /* SolveError::InvalidInput */
#define WITHIN_ERR_BUILD 2           /* BuildError: validation (empty, mismatch, weights, DOF span) */
#define WITHIN_ERR_UNSCALABLE 3      /* BuildError::UnscalableComponent */
#define WITHIN_ERR_SINGULAR 4        /* BuildError::SingularDiagonal */
#define WITHIN_ERR_INDEFINITE 5      /* mlsmr: preconditioner not positive definite (bidiag.rs:98-111) */
#define WITHIN_ERR_DIMENSION 6       /* BuildError::PreconditionerDimensionMismatch */
#define WITHIN_ERR_CUDA 7            /* device failure (allocation, launch) */
#define WITHIN_ERR_UNSUPPORTED 8     /* request outside this build's limits */

/* PreconditionerConfig (crates/within/src/config.rs:133-157) with
 * LocalSolverConfig / ApproxCholConfig / ApproxSchurConfig / ScalingConfig. */
#define WITHIN_PRECOND_OFF 0
#define WITHIN_PRECOND_ADDITIVE 1
#define WITHIN_PRECOND_DIAGONAL 2
typedef struct {
    int32_t kind;                 /* WITHIN_PRECOND_* */
    uint64_t approx_chol_seed;    /* ApproxCholConfig.seed (config.rs:20-26) */
    uint32_t approx_chol_split;   /* ApproxCholConfig.split_merge, 0 = None */
    int32_t schur_exact;          /* SchurMode::Exact (config.rs:46-59) */
    uint64_t schur_seed;          /* ApproxSchurConfig.seed */
    uint32_t schur_split;         /* ApproxSchurConfig.split (>= 1) */
    uint64_t dense_threshold;     /* LocalSolverConfig.dense_threshold (default 24) */
    double scaling_tolerance;     /* ScalingConfig.tolerance (default 1e-9) */
    uint64_t scaling_max_sweeps;  /* ScalingConfig.max_sweeps (default 2048) */
    int32_t scaling_error;        /* ScalingFailure::Error (1) or ::Warn (0) */
    int32_t reduction;            /* ReductionStrategy; accepted, the GPU combine is always a
                                     deterministic gather (schwarz/planning.rs:48-152) */
} within_precond_config;

/* LsmrOptions (config.rs:159-178) */
typedef struct {
    double tol;                   /* default 1e-8 */
    uint64_t maxiter;             /* default 1000 */
    uint64_t local_size;          /* 0 = None (no windowed reorthogonalisation) */
} within_lsmr_options;

/* Arithmetic of the operator and preconditioner applies. */
#define WITHIN_PRECISION_FP64 0      /* everything FP64 (the reference's arithmetic) */
#define WITHIN_PRECISION_MIXED 1     /* FP32 applies inside FP64 iterative refinement */

/* Per-RHS outcome: SolveResult fields (solver.rs:205-242). */
typedef struct {
    int32_t converged;
    uint64_t iterations;          /* LSMR iterations (summed over refinement sweeps) */
    double residual;              /* relative normal-equation residual estimate */
    double time_total, time_setup, time_solve;   /* seconds */
} within_solve_stats;

typedef struct within_design within_design;
typedef struct within_solver within_solver;
typedef struct within_preconditioner within_preconditioner;

/* ---- defaults ---- */
/* PreconditionerConfig::default() / LsmrOptions::default() */
void within_precond_config_default(within_precond_config* cfg);
void within_lsmr_options_default(within_lsmr_options* opts);

/* ---- design: crates/within/src/domain.rs, solver.rs:26-60 ---- */

/* IntoDesign for ArrayView2<u32> (solver.rs:34-48): codes is n_obs x n_factors,
 * column-major (F order), intercept-only factors, n_levels = max+1. */
int within_design_from_categories(const uint32_t* codes, uint64_t n_obs, uint64_t n_factors,
                                  within_design** out);
/* Design::new(Vec<Effect>) (domain.rs:155-171, effect.rs:12-42): effect e has
 * level codes levels[e] (n_obs each), an intercept flag and n_slopes[e] slope
 * columns slopes[s] taken consecutively from the flat `slopes` pointer array. */
int within_design_from_effects(uint64_t n_obs, uint64_t n_effects, const uint32_t* const* levels,
                               const int32_t* intercept, const uint64_t* n_slopes,
                               const double* const* slopes, within_design** out);
void within_design_free(within_design* d);
uint64_t within_design_n_obs(const within_design* d);
uint64_t within_design_n_dofs(const within_design* d);

/* ---- solver: crates/within/src/solver.rs:295-593 ---- */

/* Solver::new (solver.rs:361-411).  weights (host, caller order) may be NULL;
 * cfg NULL = PreconditionerInput::Default; prebuilt non-NULL =
 * PreconditionerInput::Prebuilt (its DOF count must match).  device < 0 picks
 * the current device.  The design is copied; it may be freed afterwards.
 * The host side of the build runs on a process-wide pool of up to 16 host
 * threads (the environment variable WITHIN_HOST_THREADS lowers that; 1 runs
 * it on the calling thread); the result does not depend on the count.  The
 * single-column workspaces and plans of the first solve are made here. */
int within_solver_new(const within_design* design, const double* weights,
                      const within_precond_config* cfg, const within_preconditioner* prebuilt,
                      int32_t device, within_solver** out);
/* Solver::new with an explicit tuning record (no counterpart in the reference,
 * whose strategy thresholds are constants, e.g. operator/design.rs:20 and
 * operator/design/scatter.rs:97): the kernel variants and the stop rules of
 * the round-parallel factor.  Every choice is a function of the design and
 * this record, so results stay bitwise reproducible.  within_tuning_default
 * fills the defaults; within_solver_new uses them (or the WITHIN_*
 * environment overrides).  within_b200.autotune writes a table of records
 * keyed on design statistics, from which the Python binding picks one. */
typedef struct {
    int32_t staged_sweep;       /* 1: staged (bulk-copy) row sweep / gather where they apply; 0: never */
    uint32_t wide_mean_len;     /* reduction plans whose segments average this many positions take wide
                                   tiles (default UINT32_MAX: never) */
    int32_t fuse_rounds;        /* 1: the short tail of elimination rounds runs as one launch */
    int32_t thread_per_segment; /* 1: one thread per segment where every segment is short */
    uint32_t core_dense_max;    /* a reduced system of at most this many vertices is inverted densely */
    double core_min_frac;       /* a large graph's rounds stop below this eliminated fraction */
    uint32_t max_rounds;        /* round budget (4x for graphs of at most core_small vertices) */
    uint32_t core_small;        /* graphs this small keep eliminating ... */
    uint32_t core_dense_late;   /* ... until this many vertices remain (then a dense core) */
    int32_t warp_ranges;        /* segmented reductions by warp ranges over a segment-start bitmap instead
                                   of block tiles: 1 (default) C^T and the adjoint's combines of
                                   single-column solves, 2 every tile plan, 0 none */
    int32_t gpu_cross_tab;      /* the additive-Schwarz set-up's cross-tabs on the GPU (sort and segment;
                                   the same bits as on the host): 1 (default) for designs of at least
                                   2^18 observations, 2 always, 0 never */
    int32_t vector_rows;        /* 1: the C back-substitution's short rows by groups of lanes (coalesced
                                   reads, a fixed tree per row) instead of one thread per row; 0 (default) */
} within_tuning;
void within_tuning_default(within_tuning* t);
int within_solver_new_tuned(const within_design* design, const double* weights,
                            const within_precond_config* cfg, const within_preconditioner* prebuilt,
                            int32_t device, const within_tuning* tuning, within_solver** out);
void within_solver_free(within_solver* s);
uint64_t within_solver_n_obs(const within_solver* s);
uint64_t within_solver_n_dofs(const within_solver* s);
/* Solver::warnings (solver.rs:415-417): number of BuildWarnings */
uint64_t within_solver_n_warnings(const within_solver* s);
/* SolveResult::unidentified: (term, level, column) triples; returns the count */
uint64_t within_solver_unidentified(const within_solver* s, uint64_t* triples, uint64_t cap);
/* CoefficientLayout (solver.rs:125-200): per term n_levels, offset, n_columns */
uint64_t within_solver_n_terms(const within_solver* s);
int within_solver_term_layout(const within_solver* s, uint64_t term, uint64_t* n_levels,
                              uint64_t* offset, uint64_t* n_columns);
/* Design::obs_perm (domain.rs:150-152): internal position -> caller index.
 * Returns 1 and fills out (n_obs) when the design was locality-sorted, else 0. */
int within_solver_obs_perm(const within_solver* s, uint32_t* out);
/* Solver::preconditioner (solver.rs:579-582): a shared handle, NULL when the
 * solver runs unpreconditioned.  Free it with within_preconditioner_free. */
within_preconditioner* within_solver_preconditioner(const within_solver* s);
/* Select the precision of subsequent solves (default WITHIN_PRECISION_FP64). */
int within_solver_set_precision(within_solver* s, int32_t precision);

/* Solver::solve (solver.rs:503-527): host y (caller order) -> host x (n_dofs,
 * term-major, user parametrisation) and host demeaned (n_obs, caller order).
 * Either output pointer may be NULL. */
int within_solver_solve(within_solver* s, const double* y, const within_lsmr_options* opts,
                        double* x_out, double* demeaned_out, within_solve_stats* stats);
/* Solver::solve_batch (solver.rs:530-577): Y is n_obs x k column-major on the
 * host; all k columns advance together through one multi-RHS LSMR that reads
 * the design once per apply for every column.  stats has k entries. */
int within_solver_solve_batch(within_solver* s, const double* Y, uint64_t k,
                              const within_lsmr_options* opts, double* X_out, double* D_out,
                              within_solve_stats* stats);
/* Device-resident variant of solve_batch: Y_dev, X_dev, D_dev are device
 * buffers (same layouts); stream NULL = the solver's stream. */
int within_solver_solve_batch_device(within_solver* s, const double* Y_dev, uint64_t k,
                                     const within_lsmr_options* opts, double* X_dev,
                                     double* D_dev, within_solve_stats* stats, void* stream);

/* MlsmrOptions warm start and escalation (crates/schwarz-precond/src/lsmr.rs:
 * 83-171, 206-297) on the FP64 solve of a design without slope terms.
 * x0_dev (NULL = cold) is a device warm start in x's layout (n_dofs x k
 * column-major): the solve runs on b - A x0 with the tolerances relative to
 * the original ||b|| and returns x0 + the correction; b - A x0 = 0 returns x0
 * at once (WITHIN_STOP_WARM_START_EXACT).  stale_window > 0 ends a column
 * after that many consecutive iterations whose relative normal-equation
 * residual shrank by less than stale_threshold (in [0, 1)) per iteration
 * (Staleness, lsmr.rs:95-153): converged = 0, WITHIN_STOP_ESCALATED, x the
 * iterate so far -- the warm start of the next rung of a preconditioner
 * ladder.  stop_reason (k entries, may be NULL) receives the
 * LsmrStopReason of each column (lsmr.rs:54-73). */
#define WITHIN_STOP_ZERO_RHS 0
#define WITHIN_STOP_INITIAL_NORMAL_RESIDUAL_ZERO 1
#define WITHIN_STOP_RESIDUAL_TOLERANCE 2
#define WITHIN_STOP_NORMAL_EQUATION_TOLERANCE 3
#define WITHIN_STOP_WARM_START_EXACT 4
#define WITHIN_STOP_MAX_ITERATIONS 5
#define WITHIN_STOP_ESCALATED 6
typedef struct {
    const double* x0_dev;
    uint64_t stale_window;
    double stale_threshold;
} within_solve_ext;
int within_solver_solve_batch_device_ext(within_solver* s, const double* Y_dev, uint64_t k,
                                         const within_lsmr_options* opts, const within_solve_ext* ext,
                                         double* X_dev, double* D_dev, within_solve_stats* stats,
                                         int32_t* stop_reason, void* stream);

/* One-shot solve / solve_batch (solver.rs:611-646): Solver::new + solve. */
int within_solve(const within_design* design, const double* y, const double* weights,
                 const within_lsmr_options* opts, const within_precond_config* cfg,
                 double* x_out, double* demeaned_out, within_solve_stats* stats);
int within_solve_batch(const within_design* design, const double* Y, uint64_t k,
                       const double* weights, const within_lsmr_options* opts,
                       const within_precond_config* cfg, double* X_out, double* D_out,
                       within_solve_stats* stats);

/* ---- Operator trait (crates/schwarz-precond/src/lib.rs:47-57) for the design
 * operator A = W^{1/2} D of a solver (operator/design.rs:89-117), on device
 * buffers in the INTERNAL observation order. ---- */
int within_solver_operator_apply(within_solver* s, const double* x_dev, double* y_dev,
                                 void* stream);
int within_solver_operator_apply_adjoint(within_solver* s, const double* u_dev, double* y_dev,
                                         void* stream);

/* Allocation-free variant of within_solver_operator_apply_adjoint.  It has
 * no counterpart in the reference.  It serves callers that cannot allocate
 * device memory while they run -- code recording a CUDA stream capture (an
 * allocation is not capturable), runtimes that own all device memory through
 * their own arena, and latency-critical paths that cannot afford an
 * allocation's implicit synchronisation or failure.  It computes the same
 * D^T (W^{1/2} u) on device buffers in the internal observation order, but
 * the reduction's scratch (per-tile partial sums, per-split completion
 * counters) lives in one 8 MiB static device array of the library instead of
 * solver-owned memory, and the call allocates nothing.
 *  - It uses the solver's single-column tile plan, which the solver builds at
 *    construction, so the call works on a fresh solver.
 *  - A design whose reduction needs more than 8 MiB of scratch (about
 *    700,000 tiles of 2,048 observations, i.e. more than 10^9 observation x
 *    term pairs) is rejected with WITHIN_ERR_UNSUPPORTED and a message giving
 *    the size needed.
 *  - The first call on a device looks up the array's device address (with
 *    that device current) and caches it; make that first call before any
 *    stream capture that includes this entry point.  The cache lives for the
 *    process: after cudaDeviceReset (or any teardown of the device's primary
 *    context) the cached address is stale, so do not call this entry point
 *    again in that process.
 *  - Every call on a device shares the one array and leaves its contents
 *    behind; the call clears the counters it needs.  Calls that overlap on
 *    the GPU (other streams, other threads, other solvers) race on it and
 *    must be serialised by the caller.
 *  - stream NULL = the solver's stream, and the call waits for completion. */
int within_solver_operator_apply_adjoint_noalloc(within_solver* s, const double* u_dev,
                                                 double* y_dev, void* stream);

/* ---- Many independent designs (no counterpart in the reference API, which
 * solves one design per Solver; this is the multi-design batch of many small
 * and large problems, e.g. one design per group or per bootstrap draw).
 * within_solvers_new builds n Solvers (Solver::new, solver.rs:361-411) with
 * their set-up spread over `threads` host threads; weights may be NULL or
 * hold NULL entries.  On failure no solver is left allocated.
 * within_solvers_solve_batch runs Solver::solve_batch (solver.rs:530-577) of
 * every solver: Y[i] is n_obs_i x k[i] column-major on the host, X[i] / D[i]
 * receive x and the demeaned columns (X or D NULL, or entries NULL, to skip),
 * stats[i] k[i] entries.  `threads` host threads each drive one design at a
 * time on that design's own stream, so the designs' device work overlaps;
 * every design keeps its own per-column convergence. ---- */
int within_solvers_new(uint64_t n, const within_design* const* designs, const double* const* weights,
                       const within_precond_config* cfg, int32_t device, uint32_t threads,
                       within_solver** out);
int within_solvers_solve_batch(uint64_t n, within_solver* const* solvers, const double* const* Y,
                               const uint64_t* k, const within_lsmr_options* opts, double* const* X,
                               double* const* D, within_solve_stats* const* stats, uint32_t threads);

/* ---- Preconditioner handle (operator/schwarz.rs:115-183) ---- */
void within_preconditioner_free(within_preconditioner* p);
uint64_t within_preconditioner_n(const within_preconditioner* p);
/* "Additive" or "Diagonal" */
const char* within_preconditioner_variant_name(const within_preconditioner* p);
/* Sizes of a built preconditioner (no counterpart in the reference, whose
 * Preconditioner exposes only its dimension): the counts the per-iteration
 * algorithmic bytes of its apply are computed from.  Zeros for the diagonal
 * variant apart from n. */
typedef struct {
    uint64_t n;              /* DOFs */
    uint64_t n_subdomains;
    uint64_t n_slots;        /* local slots over all subdomains (restrict / prolong entries) */
    uint64_t nnz_c;          /* C: eliminated x kept cross-block entries */
    uint64_t nnz_ct;         /* C^T */
    uint64_t nnz_fwd, nnz_bwd;   /* approximate-Cholesky factor, forward and backward pull forms */
    uint64_t nnz_dense;      /* dense pseudo-inverse blocks of small reduced systems */
    uint64_t nnz_core;       /* dense cores of round-scheduled factors */
    uint64_t n_reduced;      /* reduced (kept + ground/cover) slots */
    uint64_t n_rounds;       /* elimination rounds of the round-scheduled factor */
} within_precond_stats;
int within_preconditioner_stats(const within_preconditioner* p, within_precond_stats* out);
/* Persisted preconditioner: Preconditioner pickling (__reduce__,
 * crates/within-py/src/config.rs:366-389; Serialize/Deserialize,
 * operator/schwarz.rs:115-183) in this library's own byte format -- the host
 * image of the diagonal or Schwarz preconditioner with a magic, a version and
 * a checksum (the reference's postcard bytes embed approx-chol's private
 * layout, so the formats are not interchangeable).  serialize: buf NULL
 * returns the size in *len; otherwise cap must hold it.  deserialize uploads
 * the image to `device` (< 0: the current device); the handle is then
 * PreconditionerInput::Prebuilt for within_solver_new on a design with the
 * same DOF count, and solves with it are bitwise those of the original. */
int within_preconditioner_serialize(const within_preconditioner* p, uint8_t* buf, uint64_t cap,
                                    uint64_t* len);
int within_preconditioner_deserialize(const uint8_t* buf, uint64_t len, int32_t device,
                                      within_preconditioner** out);
/* Preconditioner::apply: y = M^{-1} x on device buffers (n each). */
int within_preconditioner_apply(const within_preconditioner* p, const double* x_dev,
                                double* y_dev, void* stream);

/* ---- Demeaning adjoint (no counterpart in the reference, which has no
 * differentiation; it differentiates the demeaned output of Solver::solve,
 * solver.rs:468-473).  For r = demeaned(z) with weights w, a loss gradient v
 * on r pulls back through one more solve with the same solver:
 *   a = v / w            within_adjoint_rhs
 *   s = demeaned(a)      within_solver_solve_batch_device on a
 *   dL/dz = w * s,  dL/dw = -sum_columns r * (a - s)   within_demean_vjp
 * Device buffers are column-major (n, k); w NULL means unit weights (then
 * a = v); the weights must be positive.  grad_z / grad_w may be NULL to skip
 * them (r and a are then not read for grad_w).  Asynchronous on `stream`. */
int within_adjoint_rhs(uint64_t n, uint64_t k, const double* v_dev, const double* w_dev,
                       double* a_dev, void* stream);
int within_demean_vjp(uint64_t n, uint64_t k, const double* r_dev, const double* a_dev,
                      const double* s_dev, const double* w_dev, double* grad_z_dev,
                      double* grad_w_dev, void* stream);

/* ---- diagnostics ---- */
const char* within_last_error(void);
/* Kernel launches issued by this library on the calling thread since the last
 * reset (graph replays count every kernel node they run). */
uint64_t within_launch_count(void);
void within_launch_count_reset(void);

#ifdef __cplusplus
}
#endif
#endif /* WITHIN_GPU_H */
