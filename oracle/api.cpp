// api.cpp -- C entry points of the CPU FP64 restatement (see within_oracle.h).
// Solver::new / solve_rhs follow crates/within/src/solver.rs:361-491.
// TEST INFRASTRUCTURE ONLY.
#include "within_oracle.h"
#include "oracle_core.hpp"

#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>

using namespace orc;

static thread_local std::string g_err;

struct or_solver {
    Design design;
    std::vector<double> sqrt_w;  // empty = unweighted
    std::unique_ptr<Preconditioner> precond;
    SlopeReparam reparam;
    size_t n_warnings = 0;
};

namespace {
struct OpView : LinOp {  // DesignOperator (operator/design.rs:22-117)
    const or_solver* s;
    explicit OpView(const or_solver* s_) : s(s_) {}
    size_t nrows() const override { return s->design.n_obs; }
    size_t ncols() const override { return s->design.n_dofs; }
    void apply(const double* x, double* y) const override {
        gather_apply(s->design, x, y, s->sqrt_w.empty() ? nullptr : s->sqrt_w.data());
    }
    void apply_adjoint(const double* u, double* y) const override {
        scatter_apply(s->design, u, s->sqrt_w.empty() ? nullptr : s->sqrt_w.data(), y);
    }
};

struct DenseOp : LinOp {
    size_t r, c;
    const double* a;
    size_t nrows() const override { return r; }
    size_t ncols() const override { return c; }
    void apply(const double* x, double* y) const override {
        for (size_t i = 0; i < r; ++i) {
            double s = 0;
            for (size_t j = 0; j < c; ++j) s += a[i * c + j] * x[j];
            y[i] = s;
        }
    }
    void apply_adjoint(const double* u, double* x) const override {
        for (size_t j = 0; j < c; ++j) {
            double s = 0;
            for (size_t i = 0; i < r; ++i) s += a[i * c + j] * u[i];
            x[j] = s;
        }
    }
};
struct DiagOp : LinOp {
    const double* d;
    size_t n;
    size_t nrows() const override { return n; }
    size_t ncols() const override { return n; }
    void apply(const double* x, double* y) const override {
        for (size_t i = 0; i < n; ++i) y[i] = d[i] * x[i];
    }
    void apply_adjoint(const double* x, double* y) const override { apply(x, y); }
};

template <class F>
int guarded(F f) {
    try {
        f();
        return 0;
    } catch (const Error& e) {
        g_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 99;
    }
}
double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

extern "C" {

const char* or_last_error(void) { return g_err.c_str(); }
void or_set_threads(int t) { orc::g_threads = t < 1 ? 1 : t; }

void or_stable_argsort(const uint32_t* key, size_t n_obs, size_t n_levels, uint32_t* perm) {
    stable_argsort(key, n_obs, n_levels, perm);
}

int or_solver_new(size_t n_obs, size_t n_terms, const uint32_t* codes, const int* intercept,
                  const size_t* n_slopes, const size_t* slope_idx, size_t n_slope_cols,
                  const double* slopes, const double* weights, const or_precond_cfg* cfg,
                  or_solver** out) {
    *out = nullptr;
    return guarded([&] {
        auto s = std::make_unique<or_solver>();
        s->design = build_design(n_obs, n_terms, codes, intercept, n_slopes, slope_idx,
                                 n_slope_cols, slopes);
        // Design::validate_weights (domain.rs:261-279)
        std::vector<double> w;
        if (weights) {
            for (size_t i = 0; i < n_obs; ++i)
                if (!(weights[i] >= 0.0 && std::isfinite(weights[i])))
                    throw Error(E_BUILD, "weight at index " + std::to_string(i) +
                                             " must be finite and non-negative");
            w.resize(n_obs);
            const auto& perm = s->design.obs_perm;
            for (size_t i = 0; i < n_obs; ++i) w[i] = perm.empty() ? weights[i] : weights[perm[i]];
        }
        s->reparam = build_reparam(s->design, weights ? w.data() : nullptr);
        PrecondCfg pc;
        if (cfg) {
            pc.kind = cfg->kind;
            pc.exact_local = cfg->exact_local != 0;
            pc.ac_seed = cfg->ac_seed;
            pc.ac_split = cfg->ac_split;
            pc.schur_exact = cfg->schur_exact != 0;
            pc.schur_seed = cfg->schur_seed;
            pc.schur_split = cfg->schur_split ? cfg->schur_split : 1;
            pc.dense_threshold = cfg->dense_threshold;
            pc.scaling_tol = cfg->scaling_tol;
            pc.scaling_max_sweeps = cfg->scaling_max_sweeps;
            pc.scaling_error = cfg->scaling_error != 0;
        }
        BuildOut b = build_preconditioner(s->design, weights ? w.data() : nullptr, pc);
        s->precond.reset(b.precond);
        s->n_warnings = b.n_warnings;
        if (weights) {
            s->sqrt_w = w;
            for (auto& v : s->sqrt_w) v = std::sqrt(v);
        }
        *out = s.release();
    });
}

void or_solver_free(or_solver* s) { delete s; }
size_t or_solver_n_dofs(const or_solver* s) { return s->design.n_dofs; }
size_t or_solver_n_obs(const or_solver* s) { return s->design.n_obs; }
size_t or_solver_n_terms(const or_solver* s) { return s->design.terms.size(); }
void or_solver_term(const or_solver* s, size_t t, size_t* nl, size_t* off, size_t* nc, int* sorted) {
    const auto& m = s->design.terms[t];
    *nl = m.n_levels;
    *off = m.offset;
    *nc = m.n_columns();
    *sorted = m.sorted ? 1 : 0;
}
int or_solver_obs_perm(const or_solver* s, uint32_t* out) {
    if (s->design.obs_perm.empty()) return 0;
    std::memcpy(out, s->design.obs_perm.data(), s->design.n_obs * sizeof(uint32_t));
    return 1;
}
int or_solver_has_precond(const or_solver* s) { return s->precond ? 1 : 0; }
size_t or_solver_n_subdomains(const or_solver* s) { return s->precond ? s->precond->n_subdomains() : 0; }
size_t or_solver_n_warnings(const or_solver* s) { return s->n_warnings; }
size_t or_solver_unidentified(const or_solver* s, size_t* triples, size_t cap) {
    const auto& u = s->reparam.unidentified;
    for (size_t i = 0; i < u.size() && i < cap; ++i) {
        triples[3 * i] = u[i].term;
        triples[3 * i + 1] = u[i].level;
        triples[3 * i + 2] = u[i].column;
    }
    return u.size();
}

int or_solver_solve(const or_solver* s, const double* y, double tol, size_t maxiter,
                    size_t local_size, double* x_out, double* demeaned_out, or_stats* st) {
    return guarded([&] {
        const Design& d = s->design;
        const size_t n = d.n_obs;
        for (size_t i = 0; i < n; ++i)
            if (!std::isfinite(y[i]))
                throw Error(E_INVALID, "response at index " + std::to_string(i) + " must be finite");
        double t0 = now();
        std::vector<double> yi(n), b(n);
        for (size_t i = 0; i < n; ++i) yi[i] = d.obs_perm.empty() ? y[i] : y[d.obs_perm[i]];
        for (size_t i = 0; i < n; ++i) b[i] = s->sqrt_w.empty() ? yi[i] : s->sqrt_w[i] * yi[i];
        double t1 = now();
        OpView op(s);
        LsmrResult r = s->precond ? mlsmr(op, b.data(), *s->precond, tol, maxiter, local_size)
                                  : lsmr(op, b.data(), tol, maxiter, local_size);
        double t2 = now();
        std::vector<double> dm(n);
        gather_apply(d, r.x.data(), dm.data(), nullptr);
        for (size_t i = 0; i < n; ++i) dm[i] = yi[i] - dm[i];
        if (s->reparam.active) s->reparam.back_transform(r.x.data());
        std::memcpy(x_out, r.x.data(), d.n_dofs * sizeof(double));
        if (d.obs_perm.empty())
            std::memcpy(demeaned_out, dm.data(), n * sizeof(double));
        else
            for (size_t k = 0; k < n; ++k) demeaned_out[d.obs_perm[k]] = dm[k];
        if (st) {
            st->converged = r.converged ? 1 : 0;
            st->iterations = r.iterations;
            st->residual = r.normal_eq_residual;
            st->residual_norm = r.residual_norm;
            st->stop_reason = r.stop_reason;
            st->time_setup = t1 - t0;
            st->time_solve = t2 - t1;
        }
    });
}

int or_solver_apply(const or_solver* s, const double* x, double* y) {
    return guarded([&] { OpView(s).apply(x, y); });
}
int or_solver_apply_adjoint(const or_solver* s, const double* u, double* y) {
    return guarded([&] { OpView(s).apply_adjoint(u, y); });
}
int or_solver_gather_plain(const or_solver* s, const double* x, double* y) {
    return guarded([&] { gather_apply(s->design, x, y, nullptr); });
}
int or_solver_precond_apply(const or_solver* s, const double* r, double* z) {
    return guarded([&] {
        if (!s->precond) {
            std::memcpy(z, r, s->design.n_dofs * sizeof(double));
            return;
        }
        s->precond->apply(r, z);
    });
}
int or_solver_loading(const or_solver* s, size_t k, double* out) {
    if (k >= s->design.loads.size()) return 1;
    std::memcpy(out, s->design.loads[k].data(), s->design.n_obs * sizeof(double));
    return 0;
}
int or_solver_sqrt_weights(const or_solver* s, double* out) {
    if (s->sqrt_w.empty()) return 0;
    std::memcpy(out, s->sqrt_w.data(), s->design.n_obs * sizeof(double));
    return 1;
}

int or_lsmr_dense(size_t rows, size_t cols, const double* a, const double* b, double tol,
                  size_t maxiter, size_t local_size, const double* precond_diag, double* x_out,
                  or_stats* st) {
    return guarded([&] {
        DenseOp op;
        op.r = rows;
        op.c = cols;
        op.a = a;
        LsmrResult r;
        if (precond_diag) {
            DiagOp m;
            m.d = precond_diag;
            m.n = cols;
            r = mlsmr(op, b, m, tol, maxiter, local_size);
        } else {
            r = lsmr(op, b, tol, maxiter, local_size);
        }
        std::memcpy(x_out, r.x.data(), cols * sizeof(double));
        if (st) {
            st->converged = r.converged;
            st->iterations = r.iterations;
            st->residual = r.normal_eq_residual;
            st->residual_norm = r.residual_norm;
            st->stop_reason = r.stop_reason;
        }
    });
}

double or_vec_norm(const double* v, size_t n) { return vec_norm(v, n); }
double or_compensated_sum(const double* v, size_t n) { return compensated_sum(v, n); }

}  // extern "C"
