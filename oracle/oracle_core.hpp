// oracle_core.hpp -- shared declarations of the CPU FP64 restatement.
// TEST INFRASTRUCTURE ONLY (see within_oracle.h).
#pragma once
#include <cstdint>
#include <cstddef>
#include <string>
#include <thread>
#include <vector>
#include <stdexcept>

namespace orc {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

enum ErrCode {
    E_INVALID = 1,      // SolveError::InvalidInput
    E_BUILD = 2,        // BuildError (validation)
    E_SCALING = 3,      // BuildError::UnscalableComponent
    E_SINGULAR = 4,     // BuildError::SingularDiagonal
    E_INDEFINITE = 5,   // mlsmr: preconditioner not positive definite
};

// Loading<u32>: -1 = Constant (intercept), k >= 0 = Covariate(k)   (domain.rs:52-77)
struct TermMeta {                     // domain.rs:79-103
    size_t n_levels = 0, offset = 0;
    bool sorted = true;
    std::vector<int> columns;
    size_t n_columns() const { return columns.size(); }
    size_t n_dofs() const { return columns.size() * n_levels; }
    size_t column_base(size_t c) const { return offset + c * n_levels; }
};

struct Design {                       // domain.rs:142-153
    size_t n_obs = 0, n_dofs = 0;
    std::vector<std::vector<uint32_t>> codes;    // per term, internal order
    std::vector<std::vector<double>> loads;      // per loading column, internal order
    std::vector<TermMeta> terms;
    std::vector<uint32_t> obs_perm;              // empty = identity
};

void stable_argsort(const uint32_t* key, size_t n_obs, size_t n_levels, uint32_t* perm);
Design build_design(size_t n_obs, size_t n_terms, const uint32_t* codes, const int* intercept,
                    const size_t* n_slopes, const size_t* slope_idx, size_t n_slope_cols,
                    const double* slopes);
void gather_apply(const Design& d, const double* src, double* dst, const double* scale);
void scatter_apply(const Design& d, const double* u, const double* sqrt_w, double* dst);

// ----- slope reparametrisation (solver/reparam.rs) -----
struct LevelTransform { std::vector<double> w, center; };
struct TermReparam {
    size_t offset = 0, n_levels = 0;
    int intercept_column = -1;
    std::vector<size_t> slope_columns;
    std::vector<LevelTransform> transforms;
    void back_transform(double* x) const;
};
struct Unidentified { size_t term, level, column; };
struct SlopeReparam {
    std::vector<TermReparam> terms;
    std::vector<Unidentified> unidentified;
    bool active = false;
    void back_transform(double* x) const { for (auto& t : terms) t.back_transform(x); }
};
SlopeReparam build_reparam(Design& d, const double* weights);

// ----- LSMR (schwarz-precond/src/lsmr*) -----
struct LinOp {
    virtual ~LinOp() {}
    virtual size_t nrows() const = 0;
    virtual size_t ncols() const = 0;
    virtual void apply(const double* x, double* y) const = 0;
    virtual void apply_adjoint(const double* x, double* y) const = 0;
};
struct LsmrResult {
    std::vector<double> x;
    bool converged = false;
    size_t iterations = 0;
    double residual_norm = 0, normal_eq_residual = 0;
    int stop_reason = 0;
};
double vec_norm(const double* v, size_t n);
double compensated_sum(const double* v, size_t n);

// Host threads of the timing mode (or_set_threads).  1 -- the default, and
// what every parity test uses -- keeps the reference's single-thread
// summation order; more threads split the row loops, reductions and SpMVs
// into contiguous ranges on std::threads (as the reference's Rayon path
// parallelises them), changing only the order of floating-point sums.
extern int g_threads;

// f(begin, end, thread) over [0, n) in g_threads contiguous ranges.
template <class F>
void par_ranges(size_t n, size_t min_n, F f) {
    const int T = g_threads;
    if (T <= 1 || n < min_n) {
        f((size_t)0, n, 0);
        return;
    }
    std::vector<std::thread> pool;
    const size_t per = (n + T - 1) / T;
    for (int t = 1; t < T; ++t) {
        const size_t a = (size_t)t * per, b = std::min(n, a + per);
        if (a >= b) break;
        pool.emplace_back([=, &f] { f(a, b, t); });
    }
    f(0, std::min(n, per), 0);
    for (auto& th : pool) th.join();
}

// sum over [0, n) of g(i): per-range partials added in range order
template <class G>
double par_sum(size_t n, size_t min_n, G g) {
    std::vector<double> part((size_t)std::max(1, g_threads), 0.0);
    par_ranges(n, min_n, [&](size_t a, size_t b, int t) {
        double s = 0.0;
        for (size_t i = a; i < b; ++i) s += g(i);
        part[t] = s;
    });
    double s = 0.0;
    for (double v : part) s += v;
    return s;
}
LsmrResult lsmr(const LinOp& a, const double* b, double tol, size_t maxiter, size_t local_size);
LsmrResult mlsmr(const LinOp& a, const double* b, const LinOp& m, double tol, size_t maxiter,
                 size_t local_size);

// ----- preconditioners -----
struct PrecondCfg {
    int kind = 1;
    bool exact_local = false;
    uint64_t ac_seed = 0;
    uint32_t ac_split = 2;
    bool schur_exact = false;
    uint64_t schur_seed = 0;
    uint32_t schur_split = 1;
    size_t dense_threshold = 24;
    double scaling_tol = 1e-9;
    size_t scaling_max_sweeps = 2048;
    bool scaling_error = false;
};

struct Preconditioner : LinOp {
    size_t n = 0;
    size_t nrows() const override { return n; }
    size_t ncols() const override { return n; }
    void apply_adjoint(const double* x, double* y) const override { apply(x, y); }
    virtual size_t n_subdomains() const { return 0; }
};

struct BuildOut {
    Preconditioner* precond = nullptr;  // nullptr = unpreconditioned
    size_t n_warnings = 0;
};
BuildOut build_preconditioner(const Design& d, const double* weights, const PrecondCfg& cfg);

}  // namespace orc
