// lsmr.cpp -- lsmr / mlsmr restated from crates/schwarz-precond/src/lsmr.rs,
// lsmr/bidiag.rs and lsmr/recurrence.rs.  Sequential FP64 (the reference's
// single-thread order).  TEST INFRASTRUCTURE ONLY.
#include "oracle_core.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <functional>

namespace orc {

// lsmr.rs:22-36 -- max-scaled norm, NaN propagating.
double vec_norm(const double* v, size_t n) {
    double scale = 0.0;
    for (size_t i = 0; i < n; ++i) scale = std::fmax(scale, std::fabs(v[i]));
    if (scale == 0.0) {
        for (size_t i = 0; i < n; ++i)
            if (std::isnan(v[i])) return NAN;
        return 0.0;
    }
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) {
        double t = v[i] / scale;
        s += t * t;
    }
    return scale * std::sqrt(s);
}

// block_elim.rs:14-29 -- Neumaier compensated sum.
double compensated_sum(const double* v, size_t n) {
    double sum = 0.0, comp = 0.0;
    for (size_t i = 0; i < n; ++i) {
        double value = v[i];
        double next = sum + value;
        if (std::fabs(sum) >= std::fabs(value))
            comp += (sum - next) + value;
        else
            comp += (value - next) + sum;
        sum = next;
    }
    return sum + comp;
}

int g_threads = 1;
constexpr size_t PAR_MIN = 65536;

static double dot(const double* a, const double* b, size_t n) {
    if (g_threads > 1) return par_sum(n, PAR_MIN, [&](size_t i) { return a[i] * b[i]; });
    double s = 0;
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}
static double axpy_with_sq_norm(double* y, const double* x, double scale, size_t n) {
    if (g_threads > 1)
        return par_sum(n, PAR_MIN, [&](size_t i) {
            double v = x[i] + scale * y[i];
            y[i] = v;
            return v * v;
        });
    double s = 0;
    for (size_t i = 0; i < n; ++i) {
        double v = x[i] + scale * y[i];
        y[i] = v;
        s += v * v;
    }
    return s;
}
static void axpby(double* y, const double* x, double alpha, double beta, size_t n) {
    par_ranges(n, PAR_MIN, [&](size_t a, size_t b, int) {
        for (size_t i = a; i < b; ++i) y[i] = alpha * x[i] + beta * y[i];
    });
}
static void scale_in_place(double* y, double s, size_t n) {
    par_ranges(n, PAR_MIN, [&](size_t a, size_t b, int) {
        for (size_t i = a; i < b; ++i) y[i] *= s;
    });
}

// bidiag.rs:98-111
static double alpha_from_vp(const double* v, const double* p, size_t n) {
    double vp = dot(v, p, n);
    if (vp < 0.0) {
        double bound = std::sqrt(DBL_EPSILON) * std::sqrt(dot(v, v, n) * dot(p, p, n));
        if (vp < -bound)
            throw Error(E_INDEFINITE, "preconditioner not positive definite (<v, Mv> < 0)");
    }
    return std::sqrt(std::max(vp, 0.0));
}

// bidiag.rs:113-217 -- window of recent basis vectors (L lanes).
struct Ring {
    size_t n = 0, cap = 0, next = 0, count = 0, lanes = 0;
    std::vector<double> buf;
    Ring(size_t m, size_t nn, size_t local_size, size_t l) : n(nn), lanes(l) {
        cap = std::min(local_size, std::min(m, nn));
        buf.assign(cap * nn * l, 0.0);
    }
    bool on() const { return cap > 0; }
    double* lane(size_t l, size_t slot) { return &buf[(l * cap + slot) * n]; }
    std::vector<size_t> chrono() const {
        std::vector<size_t> s;
        size_t start = count < cap ? 0 : next;
        for (size_t i = 0; i < count; ++i) s.push_back((start + i) % cap);
        return s;
    }
    size_t advance() {
        size_t slot = next;
        next = (next + 1) % cap;
        if (count < cap) ++count;
        return slot;
    }
};

struct Step { double alpha, beta; };

// recurrence.rs -- Givens chains, solution update, convergence test.
struct Givens {
    double c, s, r;
    Givens(double a, double b) {
        r = std::hypot(a, b);
        if (r > 0.0) { c = a / r; s = b / r; } else { c = 1.0; s = 0.0; }
    }
};
struct Rot { double rho = 1, rho_bar = 1, theta_new = 0, theta_bar = 0, zeta = 0; };



static LsmrResult run_recurrence(size_t n, Step step1, double rhs_norm, double b_norm, double tol,
                                 size_t maxiter, double* v, const std::function<Step()>& next) {
    LsmrResult res;
    // lsmr.rs:298-371
    if (step1.alpha == 0.0) {
        res.x.assign(n, 0.0);
        res.converged = true;
        res.iterations = 0;
        res.residual_norm = rhs_norm;
        res.normal_eq_residual = 0.0;
        res.stop_reason = 1;  // InitialNormalEquationResidualZero
        return res;
    }
    const double abs_tol = tol * b_norm, rel_tol = tol;
    double a_norm_sq = step1.alpha * step1.alpha;
    // LsmrRecurrenceState::init
    double alpha_bar = step1.alpha, phi_bar = step1.beta, c_bar = 1.0, s_bar = 0.0;
    double zeta_bar = step1.alpha * step1.beta;
    double zeta0 = std::max(std::fabs(zeta_bar), DBL_MIN);
    std::vector<double> x(n, 0.0), h(v, v + n), hb(n, 0.0);
    Rot prev;
    for (size_t itn = 1; itn <= maxiter; ++itn) {
        Step s = next();
        a_norm_sq += s.alpha * s.alpha + s.beta * s.beta;
        // LsmrRecurrenceState::step (recurrence.rs:81-107)
        Givens p_hat(alpha_bar, s.beta);
        double theta_new = p_hat.s * s.alpha;
        double alpha_bar_new = -p_hat.c * s.alpha;
        double phi_bar_new = p_hat.s * phi_bar;
        double theta_bar = s_bar * p_hat.r;
        Givens p_bar(c_bar * p_hat.r, theta_new);
        double zeta = p_bar.c * zeta_bar;
        double zeta_bar_new = -p_bar.s * zeta_bar;
        alpha_bar = alpha_bar_new;
        phi_bar = phi_bar_new;
        c_bar = p_bar.c;
        s_bar = p_bar.s;
        zeta_bar = zeta_bar_new;
        Rot cur{p_hat.r, p_bar.r, theta_new, theta_bar, zeta};
        // SolutionState::update (recurrence.rs:143-191)
        double t_x_den = cur.rho * cur.rho_bar;
        double t_x = std::fabs(t_x_den) > DBL_EPSILON ? cur.zeta / t_x_den : 0.0;
        double t_hb_den = prev.rho * prev.rho_bar;
        double t_hbar = std::fabs(t_hb_den) > DBL_EPSILON ? cur.theta_bar * cur.rho / t_hb_den : 0.0;
        double t_h = std::fabs(cur.rho) > DBL_EPSILON ? cur.theta_new / cur.rho : 0.0;
        for (size_t i = 0; i < n; ++i) {
            double h_old = h[i];
            double hbv = h_old - t_hbar * hb[i];
            hb[i] = hbv;
            x[i] += t_x * hbv;
            h[i] = v[i] - t_h * h_old;
        }
        // ConvergenceState::check (recurrence.rs:244-255)
        double residual = std::fabs(phi_bar);
        int stop = 0;
        if (residual <= abs_tol) {
            stop = 2;  // ResidualTolerance
        } else {
            double a_norm = std::max(std::sqrt(a_norm_sq), DBL_MIN);
            double normar = std::fabs(zeta_bar);
            if (normar / (a_norm * std::max(residual, DBL_MIN)) <= rel_tol) stop = 3;
        }
        if (stop) {
            res.x = x;
            res.converged = true;
            res.iterations = itn;
            res.residual_norm = std::fabs(phi_bar);
            res.normal_eq_residual = std::fabs(zeta_bar) / zeta0;
            res.stop_reason = stop;
            return res;
        }
        prev = cur;
    }
    res.x = x;
    res.converged = false;
    res.iterations = maxiter;
    res.residual_norm = std::fabs(phi_bar);
    res.normal_eq_residual = std::fabs(zeta_bar) / zeta0;
    res.stop_reason = 5;  // MaxIterations
    return res;
}

static void validate(const LinOp& a, const double* b, double tol) {
    if (!std::isfinite(tol) || tol < 0.0)
        throw Error(E_INVALID, "tolerance must be finite and nonnegative");
    for (size_t i = 0; i < a.nrows(); ++i)
        if (!std::isfinite(b[i]))
            throw Error(E_INVALID, "rhs entry " + std::to_string(i) + " must be finite");
}

// lsmr.rs:177-203 with GolubKahan (bidiag.rs:234-384)
LsmrResult lsmr(const LinOp& a, const double* b, double tol, size_t maxiter, size_t local_size) {
    validate(a, b, tol);
    const size_t m = a.nrows(), n = a.ncols();
    double b_norm = vec_norm(b, m);
    if (b_norm == 0.0) {
        LsmrResult r;
        r.x.assign(n, 0.0);
        r.converged = true;
        r.stop_reason = 0;  // ZeroRhs
        return r;
    }
    std::vector<double> u(m, 0.0), v(n, 0.0), av(m), atu(n);
    Ring ring(m, n, local_size, 1);
    double beta = vec_norm(b, m);
    if (beta > 0.0) {
        double inv = 1.0 / beta;
        for (size_t i = 0; i < m; ++i) u[i] = b[i] * inv;
    }
    a.apply_adjoint(u.data(), v.data());
    double alpha = std::sqrt(dot(v.data(), v.data(), n));
    if (alpha > 0.0) scale_in_place(v.data(), 1.0 / alpha, n);
    if (ring.on()) { size_t s = ring.advance(); std::copy(v.begin(), v.end(), ring.lane(0, s)); }
    Step step1{alpha, beta};
    auto next = [&]() -> Step {
        a.apply(v.data(), av.data());
        double beta_sq = axpy_with_sq_norm(u.data(), av.data(), -alpha, m);
        double bt = std::sqrt(beta_sq);
        if (bt == 0.0) {
            std::fill(v.begin(), v.end(), 0.0);
            alpha = 0.0;
            return Step{0.0, bt};
        }
        scale_in_place(u.data(), 1.0 / bt, m);
        a.apply_adjoint(u.data(), atu.data());
        double alpha_sq = axpy_with_sq_norm(v.data(), atu.data(), -bt, n);
        if (ring.on()) {
            for (size_t slot : ring.chrono()) {
                double* vj = ring.lane(0, slot);
                double c = dot(v.data(), vj, n);
                axpby(v.data(), vj, -c, 1.0, n);
            }
            alpha_sq = dot(v.data(), v.data(), n);
        }
        double al = std::sqrt(alpha_sq);
        if (al > 0.0) scale_in_place(v.data(), 1.0 / al, n);
        if (ring.on()) { size_t s = ring.advance(); std::copy(v.begin(), v.end(), ring.lane(0, s)); }
        alpha = al;
        return Step{al, bt};
    };
    return run_recurrence(n, step1, b_norm, b_norm, tol, maxiter, v.data(), next);
}

// lsmr.rs:206-295 with ModifiedGolubKahan (bidiag.rs:386-513); no warm start.
LsmrResult mlsmr(const LinOp& a, const double* b, const LinOp& mop, double tol, size_t maxiter,
                 size_t local_size) {
    validate(a, b, tol);
    const size_t m = a.nrows(), n = a.ncols();
    if (mop.nrows() != n || mop.ncols() != n)
        throw Error(E_INVALID, "preconditioner shape must match operator column count");
    double b_norm = vec_norm(b, m);
    double rhs_norm = b_norm;
    if (rhs_norm == 0.0) {
        LsmrResult r;
        r.x.assign(n, 0.0);
        r.converged = true;
        r.stop_reason = 0;
        return r;
    }
    std::vector<double> u(m, 0.0), v(n, 0.0), p(n, 0.0), av(m), atu(n);
    Ring ring(m, n, local_size, 2);
    double beta = vec_norm(b, m);
    if (beta > 0.0) {
        double inv = 1.0 / beta;
        for (size_t i = 0; i < m; ++i) u[i] = b[i] * inv;
    }
    a.apply_adjoint(u.data(), p.data());
    mop.apply(p.data(), v.data());
    double alpha = alpha_from_vp(v.data(), p.data(), n);
    if (alpha > 0.0) scale_in_place(v.data(), 1.0 / alpha, n);
    auto push = [&](double inv_alpha) {
        size_t s = ring.advance();
        std::copy(v.begin(), v.end(), ring.lane(0, s));
        double* pl = ring.lane(1, s);
        for (size_t i = 0; i < n; ++i) pl[i] = p[i] * inv_alpha;
    };
    if (ring.on()) push(alpha > 0.0 ? 1.0 / alpha : 0.0);
    double beta_prev_inv = 1.0;
    Step step1{alpha, beta};
    auto next = [&]() -> Step {
        double scale = -(alpha * beta_prev_inv);
        a.apply(v.data(), av.data());
        double beta_sq = axpy_with_sq_norm(u.data(), av.data(), scale, m);
        double bt = std::sqrt(beta_sq);
        if (bt == 0.0) {
            std::fill(v.begin(), v.end(), 0.0);
            std::fill(p.begin(), p.end(), 0.0);
            alpha = 0.0;
            beta_prev_inv = 0.0;
            return Step{0.0, bt};
        }
        double beta_inv = 1.0 / bt;
        a.apply_adjoint(u.data(), atu.data());
        double p_coeff = bt / alpha;
        axpby(p.data(), atu.data(), beta_inv, -p_coeff, n);
        mop.apply(p.data(), v.data());
        if (ring.on()) {
            for (size_t slot : ring.chrono()) {
                double* vj = ring.lane(0, slot);
                double* pj = ring.lane(1, slot);
                double c = dot(v.data(), pj, n);
                axpby(v.data(), vj, -c, 1.0, n);
                axpby(p.data(), pj, -c, 1.0, n);
            }
        }
        double an = alpha_from_vp(v.data(), p.data(), n);
        if (an > 0.0) scale_in_place(v.data(), 1.0 / an, n);
        if (ring.on()) push(an > 0.0 ? 1.0 / an : 0.0);
        alpha = an;
        beta_prev_inv = beta_inv;
        return Step{an, bt};
    };
    return run_recurrence(n, step1, rhs_norm, b_norm, tol, maxiter, v.data(), next);
}

}  // namespace orc
