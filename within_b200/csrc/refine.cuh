// refine.cuh -- mixed-precision solve: FP64 iterative refinement on the
// normal-equation residual g = D'W(z - D x) around an inner preconditioned
// conjugate-gradient solve of (D'WD) d = g whose vectors, operator data and
// preconditioner factors are stored in FP32.
//
// Why the inner solve works on the normal equations: LSMR's own residual
// r = b - A x converges to the (large) least-squares residual, so an FP32 copy
// of r carries an absolute error of ~6e-8 ||r||, whose normal component
// A^T e sets a floor of about 1e-8 on the reachable ||A^T r|| / (||A|| ||r||)
// -- exactly the accuracy asked for.  g itself is small and is formed in FP64
// from the FP64 residual, so FP32 storage costs accuracy relative to g only,
// and each refinement step reduces g by the inner tolerance with no floor
// above FP64's.  CG on D'WD is, like LSMR (MINRES on the normal equations),
// a Krylov method on A^T A with the same preconditioner.
//
// Stopping tests mirror LSMR's (recurrence.rs:193-255):
//   ||A^T r||_{M^-1} <= tol * ||A N||_F * ||r||   (normal equations)
//   ||r|| <= tol * ||b||                          (consistent system)
// with ||A^T r||_{M^-1} = sqrt(<g, M^-1 g>) (LSMR's |zeta_bar|), ||r|| (its
// |phi_bar|) formed in FP64 at every refinement step and tracked through the
// inner solve by the CG energy identity ||r_k||^2 = ||r_0||^2 - sum alpha rho,
// and ||A N||_F^2 estimated as the trace of the Lanczos matrix that CG builds
// (1/alpha_j + beta_{j-1}/alpha_{j-1} on the diagonal), which is LSMR's
// ||B_k||_F^2 (sum alpha^2 + beta^2) for the same operator.  All scalars are
// FP64; every dot product and reduction accumulates in FP64, which bounds the
// rounding of the FP32-stored sums at least as tightly as compensated FP32
// summation would.
#pragma once
#include "pdl.cuh"
#include "kernels.cuh"

namespace wgpu {

constexpr double CG_FLOOR = 1e-5;   // default inner floor: stop at this reduction of sqrt(<g, M^-1 g>)

struct CgCol {
    double rho, rho0, alpha, beta, alpha_prev, beta_prev;
    double anorm2;    // running estimate of ||A N||_F^2
    double rnorm2;    // ||r||^2 of the outer residual, tracked through the inner solve
    double bnorm;     // ||b||
    double tol;
    double floor;     // inner solve stops at this reduction of sqrt(<g, M^-1 g>)
    long long itn, inner, maxiter;
    int active;       // inner CG iterating
    int done;         // converged (or out of iterations)
    int stop;         // Stop code
    int err;
};

static_assert(sizeof(CgCol) % sizeof(double) == 0, "CgCol is addressed in doubles by the residual sweep");

// r = b - A x (FP64) and ||r||^2 per column
template <int K>
__global__ void __launch_bounds__(RED_THREADS)
k_resid64(OpParams p, const double* __restrict__ x, const double* __restrict__ b, double* __restrict__ r,
          CgCol* st, double* partials, unsigned* counter) {
    pdl_wait();
    pdl_launch_dependents();
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    const uint32_t stride = gridDim.x * blockDim.x * 4;
    for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) * 4; base < p.n; base += stride) {
        const int nr = (int)min(4u, p.n - base);
        double s[4][K];
        rows4_dx<K>(p, base, nr, x, s);
#pragma unroll
        for (int r4 = 0; r4 < 4; ++r4) {
            if (r4 >= nr) continue;
            const double w = p.sqrt_w ? __ldg(p.sqrt_w + base + r4) : 1.0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const size_t o = (size_t)(base + r4) * K + k;
                const double v = b[o] - (p.sqrt_w ? w * s[r4][k] : s[r4][k]);
                r[o] = v;
                acc[k] += v * v;
            }
        }
    }
    double tot[K];
    if (grid_reduce<K>(acc, partials, counter, tot) && threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) st[k].rnorm2 = tot[k];
}

// inner start: res = (T) g, d = 0
template <int K, class T>
__global__ void k_cg_start(uint32_t n, const double* __restrict__ g, T* __restrict__ res, T* __restrict__ d) {
    pdl_wait();
    pdl_launch_dependents();
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            res[(size_t)j * K + k] = (T)g[(size_t)j * K + k];
            d[(size_t)j * K + k] = (T)0;
        }
}

// p = z, rho0 = <res, z>, and the outer stopping tests at the FP64 residual
// first < 0: the first refinement step is the one with ctl->outer == 0.  With
// use_h, the inner loop's conditional node runs only if a column is active.
template <int K, class T>
__global__ void __launch_bounds__(RED_THREADS)
k_cg_init(uint32_t n, const T* __restrict__ res, const T* __restrict__ z, T* __restrict__ p, CgCol* st, Ctl* ctl,
          int first, double* partials, unsigned* counter, int use_h, cudaGraphConditionalHandle h_in) {
    pdl_wait();
    pdl_launch_dependents();
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const size_t o = (size_t)j * K + k;
            const T zv = z[o];
            p[o] = zv;
            acc[k] += (double)res[o] * (double)zv;
        }
    double tot[K];
    if (!grid_reduce<K>(acc, partials, counter, tot) || threadIdx.x != 0) return;
    if (first < 0) first = ctl->outer == 0 ? 1 : 0;
    bool any = false;
    for (int k = 0; k < K; ++k) {
        CgCol c = st[k];
        c.active = 0;
        if (!c.done) {
            const double rho0 = tot[k];
            const double rn = sqrt(c.rnorm2);
            if (first) c.bnorm = rn;
            if (first && rn == 0.0) {
                c.done = 1;
                c.stop = STOP_ZERO_RHS;
            } else if (rho0 < 0.0) {
                c.done = 1;
                c.err = 5;
                atomicCAS(&ctl->err, 0, 5);
            } else if (rho0 == 0.0) {
                c.done = 1;
                c.stop = first ? STOP_INIT_ZERO : STOP_NORMAL;
            } else if (!first && sqrt(rho0) <= c.tol * sqrt(c.anorm2) * rn) {
                c.done = 1;
                c.stop = STOP_NORMAL;
            } else if (!first && rn <= c.tol * c.bnorm) {
                c.done = 1;
                c.stop = STOP_RESID;
            } else if (c.itn >= c.maxiter) {
                c.done = 1;
                c.stop = STOP_MAXITER;
            } else {
                c.rho = rho0;
                c.rho0 = rho0;
                c.inner = 0;
                c.active = 1;
                any = true;
            }
        }
        st[k] = c;
    }
    ctl->all_done = any ? 0 : 1;
    ctl->k5_skip = 0;
    if (use_h) cudaGraphSetConditional(h_in, any ? 1u : 0u);
}

// End of one refinement step of the device-driven mixed solve: take another
// step while a column has not converged (at most 64 steps).
__global__ void k_outer_cond(const CgCol* st, Ctl* ctl, cudaGraphConditionalHandle h_out) {
    bool any = false;
    for (int k = 0; k < 8; ++k) any = any || !st[k].done;
    const int o = ctl->outer + 1;
    ctl->outer = o;
    cudaGraphSetConditional(h_out, (any && !ctl->err && o < 64) ? 1u : 0u);
}

// alpha = rho / <p, A^T A p>
template <int K, class T>
__global__ void __launch_bounds__(RED_THREADS)
k_cg_alpha(uint32_t n, const T* __restrict__ p, const T* __restrict__ q, CgCol* st, Ctl* ctl, double* partials,
           unsigned* counter) {
    pdl_wait();
    pdl_launch_dependents();
    if (ctl->all_done) return;
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += (double)p[(size_t)j * K + k] * (double)q[(size_t)j * K + k];
    double tot[K];
    if (!grid_reduce<K>(acc, partials, counter, tot) || threadIdx.x != 0) return;
    for (int k = 0; k < K; ++k) {
        CgCol& c = st[k];
        if (!c.active) continue;
        if (!(tot[k] > 0.0)) {   // no curvature left along p: stop this inner solve
            c.active = 0;
            c.alpha = 0.0;
            continue;
        }
        c.alpha = c.rho / tot[k];
    }
}

// d += alpha p, res -= alpha q
template <int K, class T>
__global__ void k_cg_update(uint32_t n, const T* __restrict__ p, const T* __restrict__ q, T* __restrict__ d,
                            T* __restrict__ res, const CgCol* st, const Ctl* ctl) {
    pdl_wait();
    pdl_launch_dependents();
    if (ctl->all_done) return;
    double a[K];
    bool act[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        act[k] = st[k].active != 0;
        a[k] = st[k].alpha;
    }
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!act[k]) continue;
            const size_t o = (size_t)j * K + k;
            d[o] = (T)((double)d[o] + a[k] * (double)p[o]);
            res[o] = (T)((double)res[o] - a[k] * (double)q[o]);
        }
}

// rho' = <res, z>, beta = rho' / rho, the norm estimates and the stopping tests
template <int K, class T>
__global__ void __launch_bounds__(RED_THREADS)
k_cg_beta(uint32_t n, const T* __restrict__ res, const T* __restrict__ z, CgCol* st, Ctl* ctl, double* partials,
          unsigned* counter) {
    pdl_wait();
    pdl_launch_dependents();
    if (ctl->all_done) return;
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += (double)res[(size_t)j * K + k] * (double)z[(size_t)j * K + k];
    double tot[K];
    if (!grid_reduce<K>(acc, partials, counter, tot) || threadIdx.x != 0) return;
    bool any = false;
    for (int k = 0; k < K; ++k) {
        CgCol c = st[k];
        if (c.active && c.alpha > 0.0) {
            // Lanczos diagonal entry of this step: 1/alpha_j + beta_{j-1}/alpha_{j-1}
            c.anorm2 += 1.0 / c.alpha + (c.inner > 0 ? c.beta_prev / c.alpha_prev : 0.0);
            c.rnorm2 = fmax(c.rnorm2 - c.alpha * c.rho, 0.0);
            const double rho_new = fmax(tot[k], 0.0);
            c.beta = c.rho > 0.0 ? rho_new / c.rho : 0.0;
            c.alpha_prev = c.alpha;
            c.beta_prev = c.beta;
            c.rho = rho_new;
            c.itn += 1;
            c.inner += 1;
            const double rn = sqrt(c.rnorm2);
            const double gn = sqrt(rho_new);
            if (gn <= c.floor * sqrt(c.rho0) || gn <= c.tol * sqrt(c.anorm2) * rn || rn <= c.tol * c.bnorm ||
                c.itn >= c.maxiter || rho_new == 0.0)
                c.active = 0;
        } else {
            c.active = 0;
        }
        any = any || c.active;
        st[k] = c;
    }
    ctl->all_done = any ? 0 : 1;
}

// p = z + beta p
template <int K, class T>
__global__ void k_cg_dir(uint32_t n, const T* __restrict__ z, T* __restrict__ p, const CgCol* st, const Ctl* ctl) {
    pdl_wait();
    pdl_launch_dependents();
    if (ctl->all_done) return;
    double b[K];
    bool act[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        act[k] = st[k].active != 0;
        b[k] = st[k].beta;
    }
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!act[k]) continue;
            const size_t o = (size_t)j * K + k;
            p[o] = (T)((double)z[o] + b[k] * (double)p[o]);
        }
}

// x += d (FP64 accumulation of the FP32 correction)
template <int K, class T>
__global__ void k_add_delta(uint32_t n, const T* __restrict__ d, double* __restrict__ x) {
    pdl_wait();
    pdl_launch_dependents();
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) x[(size_t)j * K + k] += (double)d[(size_t)j * K + k];
}

__global__ void k_cg_setup(CgCol* st, int k_used, double tol, long long maxiter, Ctl* ctl, double floor) {
    for (int k = 0; k < 8; ++k) {
        CgCol c;
        memset(&c, 0, sizeof(c));
        c.tol = tol;
        c.floor = floor;
        c.maxiter = maxiter;
        c.stop = STOP_NONE;
        if (k >= k_used) {
            c.done = 1;
            c.stop = STOP_ZERO_RHS;
        }
        st[k] = c;
    }
    memset(ctl, 0, sizeof(Ctl));
    ctl->bodies_left = (int)min(maxiter + 2, (long long)INT_MAX);
}

}  // namespace wgpu
