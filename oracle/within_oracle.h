/*
 * within_oracle.h -- CPU FP64 restatement of leostimpfle/within's fixed-effects
 * solve path.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and
 * the CPU-baseline leg of the benchmark call it as the checker.  Nothing in the
 * product library links or calls it.
 *
 * What it restates (reference paths are relative to the reference checkout):
 *   crates/within/src/domain.rs            Design::build, stable_argsort, permutations
 *   crates/within/src/domain/effect.rs     Effect::new validation
 *   crates/within/src/operator/design/{gather,scatter}.rs gather/scatter / scatter_apply
 *   crates/within/src/solver/reparam.rs    slope whitening + back transform
 *   crates/within/src/operator/schwarz.rs  Off / Diagonal / Additive selection
 *   crates/within/src/domain/cross_tab{,/accumulate}.rs cross-tab, components, extraction
 *   crates/within/src/domain/factor_pairs{,/sddm}.rs subdomains, SDDM conversion, PoU weights
 *   crates/within/src/block_elim/{solver,schur,factor}.rs block elimination, exact/sampled Schur
 *   crates/schwarz-precond/src/lsmr*       lsmr / mlsmr, bidiagonalisation, recurrences
 *   crates/schwarz-precond/src/{domain,local_solve}.rs   restrict / prolongate
 *
 * The reduced-system factorisation lives in the external crate approx-chol
 * 0.5.0 (crates.io, Cargo.lock:27-30), which is not vendored in the reference.
 * Its dense "ExactBelow" backend is restated here as a dense LDL^T with a
 * pseudo-inverse pivot, and its approximate backend as the published
 * Gao-Kyng-Spielman approximate Cholesky (arXiv:2303.00709, random elimination
 * order, clique-tree sampling).  Factor values are therefore parity-unpinned;
 * solutions are pinned through the exact route and the known-answer tests.
 */
#ifndef WITHIN_ORACLE_H
#define WITHIN_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* PreconditionerConfig (crates/within/src/config.rs:133-157) plus oracle routing. */
typedef struct {
    int kind;                  /* 0 Off, 1 Additive, 2 Diagonal */
    int exact_local;           /* 1: exact Schur + dense factor for every subdomain (small cases) */
    uint64_t ac_seed;          /* ApproxCholConfig.seed */
    uint32_t ac_split;         /* ApproxCholConfig.split_merge (0 = None) */
    int schur_exact;           /* SchurMode::Exact */
    uint64_t schur_seed;       /* ApproxSchurConfig.seed */
    uint32_t schur_split;      /* ApproxSchurConfig.split */
    size_t dense_threshold;    /* LocalSolverConfig.dense_threshold */
    double scaling_tol;        /* ScalingConfig.tolerance */
    size_t scaling_max_sweeps; /* ScalingConfig.max_sweeps */
    int scaling_error;         /* ScalingFailure::Error */
} or_precond_cfg;

typedef struct {
    int converged;
    size_t iterations;
    double residual;           /* relative normal-equation residual estimate */
    double residual_norm;      /* |phi_bar| */
    int stop_reason;           /* LsmrStopReason order, lsmr.rs:57-72 */
    double time_setup, time_solve;
} or_stats;

typedef struct or_solver or_solver;

const char* or_last_error(void);
void or_set_threads(int n);

/* domain.rs:110-140 */
void or_stable_argsort(const uint32_t* key, size_t n_obs, size_t n_levels, uint32_t* perm);

/*
 * Solver::new (solver.rs:361-411).  codes: n_obs x n_terms, column-major.
 * Term t has intercept[t] in {0,1} and n_slopes[t] slope columns whose indices
 * into `slopes` (n_obs x n_slope_cols, column-major) are listed consecutively in
 * slope_idx.  weights may be NULL.  cfg NULL = library default.
 */
int or_solver_new(size_t n_obs, size_t n_terms, const uint32_t* codes,
                  const int* intercept, const size_t* n_slopes, const size_t* slope_idx,
                  size_t n_slope_cols, const double* slopes, const double* weights,
                  const or_precond_cfg* cfg, or_solver** out);
void or_solver_free(or_solver* s);

size_t or_solver_n_dofs(const or_solver* s);
size_t or_solver_n_obs(const or_solver* s);
size_t or_solver_n_terms(const or_solver* s);
/* per-term layout: n_levels, offset, n_columns, sorted flag (after locality sort) */
void or_solver_term(const or_solver* s, size_t t, size_t* n_levels, size_t* offset,
                    size_t* n_columns, int* sorted);
/* obs_perm (internal -> caller index); returns 0 when no permutation was applied */
int or_solver_obs_perm(const or_solver* s, uint32_t* out);
int or_solver_has_precond(const or_solver* s);
size_t or_solver_n_subdomains(const or_solver* s);
size_t or_solver_n_warnings(const or_solver* s);
/* unidentified directions as (term, level, column) triples; returns count */
size_t or_solver_unidentified(const or_solver* s, size_t* triples, size_t cap);

/* Solver::solve (solver.rs:423-527): x in caller parametrisation, demeaned in caller order */
int or_solver_solve(const or_solver* s, const double* y, double tol, size_t maxiter,
                    size_t local_size, double* x_out, double* demeaned_out, or_stats* st);

/* Operator plumbing in the design's internal row order (design.rs:97-116). */
int or_solver_apply(const or_solver* s, const double* x, double* y);
int or_solver_apply_adjoint(const or_solver* s, const double* u, double* y);
/* gather_apply without weights (demean path, solver.rs:469-473), internal order */
int or_solver_gather_plain(const or_solver* s, const double* x, double* y);
int or_solver_precond_apply(const or_solver* s, const double* r, double* z);
/* loading column k of the internal frame (after reparametrisation) */
int or_solver_loading(const or_solver* s, size_t k, double* out);
/* sqrt weights in internal order, returns 0 if unweighted */
int or_solver_sqrt_weights(const or_solver* s, double* out);

/*
 * lsmr / mlsmr on a dense row-major operator (the reference's fixture
 * operators, lsmr/fixtures.rs).  precond_diag NULL => lsmr (GolubKahan),
 * otherwise mlsmr with M^-1 = diag(precond_diag).
 */
int or_lsmr_dense(size_t rows, size_t cols, const double* a, const double* b, double tol,
                  size_t maxiter, size_t local_size, const double* precond_diag,
                  double* x_out, or_stats* st);

double or_vec_norm(const double* v, size_t n);
double or_compensated_sum(const double* v, size_t n);

#ifdef __cplusplus
}
#endif
#endif
