// kernels.cuh -- device code of the fixed-effects solve (sm_100a).
//
// Vector layout: K right-hand sides are interleaved, element (i, k) of an
// observation vector lives at [i*K + k] and of a DOF vector at [j*K + k], so a
// thread that reads one code reads every column's coefficient from one
// contiguous K-wide run.  All reductions are formed in a fixed order (per-thread
// strided partials, a fixed shuffle tree, per-block partials summed by the last
// block in block order), so every result is bitwise reproducible.
#pragma once
#include "pdl.cuh"
#include <cfloat>
#include <climits>
#include <cstdint>

#include "segreduce.cuh"
#include "segsweep.cuh"

namespace wgpu {

constexpr int MAXQ = 8, MAXC = 4, MAXS = 16;
constexpr int RED_THREADS = 256;

// Design-operator parameters (operator/design.rs:22-62), passed by value.
// T is the storage type of the floating operands (double; float for the
// mixed-precision inner solve); sums are always formed in double.
template <class T>
struct OpParamsT {
    uint32_t n;
    int Q;
    const uint32_t* codes[MAXQ];
    uint32_t off[MAXQ], L[MAXQ];
    int ncol[MAXQ];
    int load[MAXQ][MAXC];      // -1 intercept, else loading column
    const T* loads[MAXS];
    const T* sqrt_w;           // nullptr = unweighted
};
using OpParams = OpParamsT<double>;

// Per-column LSMR scalar state (lsmr/recurrence.rs + bidiag.rs), double
// buffered by iteration parity.
struct ColState {
    double alpha, beta_prev_inv, beta;
    double alpha_bar, phi_bar, c_bar, s_bar, zeta_bar, zeta0;
    double prev_rho, prev_rho_bar;
    double a_norm_sq, abs_tol, rel_tol;
    double t_x, t_hbar, t_h, vscale;
    double b_norm;
    long long itn, maxiter;
    int done, stop, upd, err;
    // Staleness escalation (lsmr.rs:83-153): stale_window consecutive ratios
    // |zeta_bar_k| / |zeta_bar_{k-1}| above stale_thr end the column with
    // STOP_ESCALATED; window 0 = never
    double stale_thr, stale_prev;
    int stale_window, stale_n;
};

struct Ctl {
    int all_done;     // every column finished: loop kernels return at entry
    int k5_skip;      // the vector update of this iteration has nothing to do
    int err;          // first error code raised on the device
    int bodies_left;  // device-side graph loop: bodies (2 iterations each) still allowed
    int bodies_run;   // device-side graph loop: bodies executed
    int outer;        // mixed precision: refinement steps taken
    int pad[2];
};

// End of one body (two LSMR iterations) of the device-side graph loop: run
// the body again while a column is active, no error was raised and the body
// budget (set from maxiter by k_norm_b) is not spent.
__global__ void k_loop_cond(Ctl* ctl, cudaGraphConditionalHandle h) {
    const int left = ctl->bodies_left - 1;
    ctl->bodies_left = left;
    ctl->bodies_run += 1;
    cudaGraphSetConditional(h, (!ctl->all_done && !ctl->err && left > 0) ? 1u : 0u);
}

// LsmrStopReason (lsmr.rs:54-73), same order
enum Stop { STOP_NONE = -1, STOP_ZERO_RHS = 0, STOP_INIT_ZERO = 1, STOP_RESID = 2, STOP_NORMAL = 3,
            STOP_WARM_EXACT = 4, STOP_MAXITER = 5, STOP_ESCALATED = 6 };
constexpr int ERR_WARM_NONFINITE = 10;   // device error: b - A x0 has a non-finite norm

// ---------------------------------------------------------------------------
// fixed-order block reduction helpers

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// K consecutive values of an interleaved vector row into registers of type A
// (double, or float in the mixed-precision inner solve), and back:
// one 16-byte access per 16 bytes of the row (rows are 16-byte aligned
// whenever they are 16 bytes or longer).
template <int K, class T, class A>
__device__ __forceinline__ void ldk(const T* p, A (&v)[K]) {
    if constexpr (sizeof(T) == 8 && K % 2 == 0) {
#pragma unroll
        for (int i = 0; i < K / 2; ++i) {
            const double2 q = reinterpret_cast<const double2*>(p)[i];
            v[2 * i] = q.x;
            v[2 * i + 1] = q.y;
        }
    } else if constexpr (sizeof(T) == 4 && K % 4 == 0) {
#pragma unroll
        for (int i = 0; i < K / 4; ++i) {
            const float4 q = reinterpret_cast<const float4*>(p)[i];
            v[4 * i] = q.x;
            v[4 * i + 1] = q.y;
            v[4 * i + 2] = q.z;
            v[4 * i + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = (A)p[k];
    }
}

// ldk through the read-only path (data no thread of the kernel writes)
template <int K, class T, class A>
__device__ __forceinline__ void ldgk(const T* __restrict__ p, A (&v)[K]) {
    if constexpr (sizeof(T) == 8 && K % 2 == 0) {
#pragma unroll
        for (int i = 0; i < K / 2; ++i) {
            const double2 q = __ldg(reinterpret_cast<const double2*>(p) + i);
            v[2 * i] = q.x;
            v[2 * i + 1] = q.y;
        }
    } else if constexpr (sizeof(T) == 4 && K % 4 == 0) {
#pragma unroll
        for (int i = 0; i < K / 4; ++i) {
            const float4 q = __ldg(reinterpret_cast<const float4*>(p) + i);
            v[4 * i] = q.x;
            v[4 * i + 1] = q.y;
            v[4 * i + 2] = q.z;
            v[4 * i + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = (A)__ldg(p + k);
    }
}

template <int K, class T, class A>
__device__ __forceinline__ void stk(T* p, const A (&v)[K]) {
    if constexpr (sizeof(T) == 8 && K % 2 == 0) {
#pragma unroll
        for (int i = 0; i < K / 2; ++i) reinterpret_cast<double2*>(p)[i] = make_double2(v[2 * i], v[2 * i + 1]);
    } else if constexpr (sizeof(T) == 4 && K % 4 == 0) {
#pragma unroll
        for (int i = 0; i < K / 4; ++i)
            reinterpret_cast<float4*>(p)[i] =
                make_float4((float)v[4 * i], (float)v[4 * i + 1], (float)v[4 * i + 2], (float)v[4 * i + 3]);
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) p[k] = (T)v[k];
    }
}

// Column i of a [nblk][stride] table of block partials, summed in one fixed
// order by a whole warp: lane l adds rows l, l+32, ..., then a fixed shuffle
// tree; every lane returns the total.
__device__ __forceinline__ double warp_col_sum(const double* part, unsigned nblk, size_t stride, size_t i) {
    const int lane = threadIdx.x & 31;
    double a = 0.0;
    for (unsigned blk = lane; blk < nblk; blk += 32) a += __ldcg(&part[(size_t)blk * stride + i]);
    return warp_sum(a);
}

// Publishes NV block partials and returns true in the (single) last block to
// finish, in which `tot` (thread 0) holds the grand totals summed in block
// order.  All NV values share one barrier round, and the last block loads
// the partials of every value in one pass, so its loads overlap instead of
// running NV dependent passes; each value's additions keep the order of a
// per-value block_sum.
template <int NV>
__device__ bool grid_reduce(const double (&v)[NV], double* partials, unsigned* counter,
                            double (&tot)[NV]) {
    __shared__ double sm[NV][32];
    __shared__ int is_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const double x = warp_sum(v[i]);
        if (lane == 0) sm[i][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double t = 0;
            for (int w = 0; w < nw; ++w) t += sm[i][w];
            partials[(size_t)blockIdx.x * NV + i] = t;
        }
        __threadfence();
        unsigned prev = atomicAdd(counter, 1u);
        is_last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double a[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) a[i] = 0.0;
    for (unsigned blk = threadIdx.x; blk < gridDim.x; blk += blockDim.x)
#pragma unroll
        for (int i = 0; i < NV; ++i) a[i] += __ldcg(&partials[(size_t)blk * NV + i]);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const double x = warp_sum(a[i]);
        if (lane == 0) sm[i][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double t = 0;
            for (int w = 0; w < nw; ++w) t += sm[i][w];
            tot[i] = t;
        }
        *counter = 0;
    }
    return true;
}

// ---------------------------------------------------------------------------
// D x rows (gather.rs:10-109): term sums accumulate in term order from 0.
// D x for 4 consecutive observations [base, base+nr) per call: the code loads
// are one 16-byte vector per term, for K >= 2 the codes of the first DX_QR
// terms are all requested before any coefficient gather (at K = 1 the extra
// registers cost more occupancy than the overlap gains: 2.66 vs 2.83 TB/s on
// the 10M-row panel), and all gathers of the 4 rows are independent, so a
// thread keeps several memory requests in flight.
constexpr int DX_QR = 3;

__device__ __forceinline__ void load_codes4(const uint32_t* __restrict__ c, uint32_t base, int nr,
                                            uint32_t (&code)[4]) {
    if (nr == 4) {
        const uint4 c4 = __ldg(reinterpret_cast<const uint4*>(c + base));
        code[0] = c4.x; code[1] = c4.y; code[2] = c4.z; code[3] = c4.w;
    } else {
#pragma unroll
        for (int r = 0; r < 4; ++r) code[r] = r < nr ? __ldg(c + base + r) : 0u;
    }
}

template <int K, class T = double>
__device__ __forceinline__ void rows4_dx(const OpParamsT<T>& p, uint32_t base, int nr,
                                         const T* __restrict__ x, double (&s)[4][K]) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int k = 0; k < K; ++k) s[r][k] = 0.0;
    constexpr int QR = K == 1 ? 1 : DX_QR;
    uint32_t cq[QR][4];
#pragma unroll
    for (int t = 0; t < QR; ++t)
        if (t < p.Q) load_codes4(p.codes[t], base, nr, cq[t]);
    for (int t = 0; t < p.Q; ++t) {
        uint32_t code[4];
        if (t < QR) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                uint32_t c = cq[0][r];
#pragma unroll
                for (int q = 1; q < QR; ++q)
                    if (t == q) c = cq[q][r];
                code[r] = c;
            }
        } else {
            load_codes4(p.codes[t], base, nr, code);
        }
        for (int c = 0; c < p.ncol[t]; ++c) {
            const size_t col = (size_t)p.off[t] + (size_t)c * p.L[t];
            const int li = p.load[t][c];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (r >= nr) continue;
                const double ld = li < 0 ? 1.0 : (double)__ldg(p.loads[li] + base + r);
                double xg[K];
                ldgk<K, T>(x + (col + code[r]) * K, xg);
#pragma unroll
                for (int k = 0; k < K; ++k) s[r][k] += xg[k] * ld;
            }
        }
    }
}

// y = W^{1/2} D x  (Operator::apply; internal order)
template <int K, class T = double>
__global__ void k_apply(OpParamsT<T> p, const T* __restrict__ x, T* __restrict__ y, const int* skip = nullptr) {
    pdl_wait();
    pdl_launch_dependents();
    if (skip && *skip) return;
    const uint32_t stride = gridDim.x * blockDim.x * 4;
    for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) * 4; base < p.n; base += stride) {
        const int nr = (int)min(4u, p.n - base);
        double s[4][K];
        rows4_dx<K, T>(p, base, nr, x, s);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (r >= nr) continue;
            const double w = p.sqrt_w ? (double)p.sqrt_w[base + r] : 1.0;
#pragma unroll
            for (int k = 0; k < K; ++k) y[(size_t)(base + r) * K + k] = (T)(p.sqrt_w ? w * s[r][k] : s[r][k]);
        }
    }
}

// demeaned = y - D x (unweighted; solver.rs:468-473)
template <int K>
__global__ void k_demean(OpParams p, const double* __restrict__ x, const double* __restrict__ yint,
                         double* __restrict__ out) {
    pdl_wait();
    pdl_launch_dependents();
    const uint32_t stride = gridDim.x * blockDim.x * 4;
    for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) * 4; base < p.n; base += stride) {
        const int nr = (int)min(4u, p.n - base);
        double s[4][K];
        rows4_dx<K>(p, base, nr, x, s);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (r >= nr) continue;
            double o[K];
            ldk<K, double>(yint + (size_t)(base + r) * K, o);
#pragma unroll
            for (int k = 0; k < K; ++k) o[k] -= s[r][k];
            stk<K, double>(out + (size_t)(base + r) * K, o);
        }
    }
}

// LSMR step, first half (bidiag.rs:278-283): u <- A v + scale u with
// scale = -(alpha / beta_prev), beta = ||u||; fused in one row sweep.
template <int K>
__global__ void __launch_bounds__(RED_THREADS)
k_gather_update(OpParams p, const double* __restrict__ v, double* __restrict__ u, ColState* cur,
                Ctl* ctl, double* partials, unsigned* counter) {
    pdl_wait();
    pdl_launch_dependents();
    if (ctl->all_done) {
        // nothing left to update this iteration either (k_alpha_step also returns)
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->k5_skip = 1;
        return;
    }
    double scale[K];
    bool act[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        act[k] = !cur[k].done;
        scale[k] = -(cur[k].alpha * cur[k].beta_prev_inv);
    }
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    const uint32_t stride = gridDim.x * blockDim.x * 4;
    for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) * 4; base < p.n; base += stride) {
        const int nr = (int)min(4u, p.n - base);
        double s[4][K];
        rows4_dx<K>(p, base, nr, v, s);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (r >= nr) continue;
            const double w = p.sqrt_w ? __ldg(p.sqrt_w + base + r) : 1.0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const double av = p.sqrt_w ? w * s[r][k] : s[r][k];
                double* up = u + (size_t)(base + r) * K + k;
                const double nu = act[k] ? av + scale[k] * (*up) : *up;
                if (act[k]) *up = nu;
                acc[k] += nu * nu;
            }
        }
    }
    double tot[K];
    if (grid_reduce<K>(acc, partials, counter, tot) && threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (act[k]) cur[k].beta = sqrt(tot[k]);
    }
}

// ---------------------------------------------------------------------------
// Scatter D^T (W^{1/2} u) as a segmented reduction (scatter.rs:14-73): one
// problem per (term, coefficient column); segments are the term's levels,
// positions its level-sorted observation order (identity when sorted).
struct ScatterProb {
    const uint32_t* seg_ptr;   // level_ptr (n_levels + 1)
    const uint32_t* order;     // position -> observation, or -> run (nullptr = identity)
    const double* load;        // loading column (nullptr = intercept)
    const float* load_f;       // the same column in float (mixed-precision inner solve)
    uint32_t out_off;          // DOF of level 0 of this column
    uint32_t ncol;             // run-sum problems: columns of the term
    const double* run_sum;     // non-null: positions are runs, values run_sum[(run*ncol+col)*K+k]
    uint32_t col;              // run-sum problems: this problem's column
    uint32_t pad;
};

// EPI 0: out = sum (Operator::apply_adjoint)
// EPI 1: p~ <- sum / beta - (beta / alpha) p~ (bidiag.rs:474-485), per column,
//        skipping finished columns; beta == 0 (lucky breakdown) zeroes p~.
template <int K, int EPI, class T = double>
struct ScatterF {
    using Prob = ScatterProb;
    using Acc = double;
    const ScatterProb* probs;
    const T* u;
    const T* sqrt_w;
    T* out;
    const ColState* cur;
    __device__ const uint32_t* seg_ptr(const Prob& pr) const { return pr.seg_ptr; }
    __device__ void value(const Prob& pr, uint32_t pos, double (&v)[K]) const {
        const uint32_t i = pr.order ? __ldg(pr.order + pos) : pos;
        if (pr.run_sum) {   // combine of run sums formed by the row sweep (rowsweep.cuh)
            const double* rs = pr.run_sum + ((size_t)i * pr.ncol + pr.col) * K;
#pragma unroll
            for (int k = 0; k < K; ++k) v[k] = __ldg(rs + k);
            return;
        }
        double f = 1.0;
        if constexpr (sizeof(T) == 8) {
            if (pr.load) f = __ldg(pr.load + i);
        } else {
            if (pr.load_f) f = (double)__ldg(pr.load_f + i);
        }
        if (sqrt_w) f *= (double)__ldg(sqrt_w + i);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = 0.0;
        ldk<K, T>(u + (size_t)i * K, v);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] *= f;
    }
    __device__ void emit(const Prob& pr, uint32_t seg, const double (&s)[K]) const {
        T* o = out + ((size_t)pr.out_off + seg) * K;
        if (EPI == 0) {
#pragma unroll
            for (int k = 0; k < K; ++k) o[k] = (T)s[k];
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (cur[k].done) continue;
                const double beta = cur[k].beta;
                o[k] = beta == 0.0 ? 0.0 : s[k] * (1.0 / beta) - (beta / cur[k].alpha) * o[k];
            }
        }
    }
};

// ---------------------------------------------------------------------------
// Additive Schwarz apply (schwarz-precond executor.rs + block_elim/solver.rs),
// all subdomains at once.  See SchwarzHost (host.hpp) for the layout.
template <class T>
struct SchwarzDevT {
    uint32_t n_sub;
    const uint32_t* loc_ptr;
    const uint32_t* n_elim;
    const uint32_t* red_off;
    const uint32_t* n_kept;
    const uint32_t* red_n;
    const int* mode;
    const uint32_t* glob;
    const T* scale;
    const uint32_t* slot_sub;
    const T* inv_e;
    const uint32_t* ct_col;
    const T* ct_val;       // C^T / D_e
    const T* ct_rowsum;
    const uint32_t* ct_row_slot;
    const uint32_t* ct_row_red;
    const uint32_t* elim_slot;
    const uint32_t* c_col;
    const T* c_val;
    const uint32_t* red_sub;
    const uint32_t* dense_row_slot;
    const uint32_t* dense_col;
    const T* dense_val;
    const T* dinv;
    const uint32_t* fwd_row;
    const uint32_t* fwd_col;
    const T* fwd_val;
    const uint32_t* bwd_row;
    const uint32_t* bwd_col;
    const T* bwd_val;
    const uint32_t* dof_slot;
    const uint32_t* kept_ptr;
    const uint32_t* core_row_slot;
    const uint32_t* core_col;
    const T* core_val;
    // work (K-interleaved)
    T* rl;   // restricted, folded local rhs (per local slot)
    T* sl;   // local solution (per local slot)
    T* rb;   // reduced rhs
    T* yv;   // forward-substitution values
    T* xv;   // reduced solution
    T* m1;   // per subdomain: mean of rl (floating) else 0
    T* m2;   // per subdomain: mean of the reduced rhs (floating) else 0
    T* m3;   // per subdomain: mean of the local solution (floating) else 0
};
using SchwarzDev = SchwarzDevT<double>;

struct SegProb {          // generic: one pointer array + a segment base
    const uint32_t* seg_ptr;
    uint32_t seg_base;    // added to the local segment id
    uint32_t pad;
};

// solution of kept index k (reduced slot u) after the gauge / cover read-back
template <int K, class T = double>
__device__ __forceinline__ void kept_solution(const SchwarzDevT<T>& S, uint32_t u, T (&o)[K]) {
    const uint32_t s = S.red_sub[u];
    const int m = S.mode[s];
    ldk<K, T>(S.xv + (size_t)u * K, o);
    if (m != 0) {
        T q[K];
        if (m == 1) {
            ldk<K, T>(S.xv + (size_t)(S.red_off[s] + S.n_kept[s]) * K, q);
#pragma unroll
            for (int k = 0; k < K; ++k) o[k] = o[k] - q[k];
        } else {
            ldk<K, T>(S.xv + (size_t)(u + S.n_kept[s]) * K, q);
#pragma unroll
            for (int k = 0; k < K; ++k) o[k] = (T)0.5 * (o[k] - q[k]);
        }
    }
}

// S1: restrict + fold, per-subdomain sums -> m1 (solver.rs:445-451, domain.rs:133-152)
template <int K, class T = double>
struct RestrictF {
    using Prob = SegProb;
    using Acc = T;   // sums in the storage type (FP32 in the mixed-precision inner solve)
    const SegProb* probs;
    SchwarzDevT<T> S;
    const T* r;
    __device__ const uint32_t* seg_ptr(const Prob& p) const { return p.seg_ptr; }
    __device__ void value(const Prob&, uint32_t j, T (&v)[K]) const {
        const uint32_t g = __ldg(S.glob + j);
        const T sc = __ldg(S.scale + j);
        ldk<K, T>(r + (size_t)g * K, v);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] *= sc;
        stk<K, T>(S.rl + (size_t)j * K, v);
    }
    __device__ void emit(const Prob& p, uint32_t seg, const T (&s)[K]) const {
        const uint32_t sub = p.seg_base + seg;
        const bool fl = S.mode[sub] == 0;
        const T inv = 1.0 / (double)(S.loc_ptr[sub + 1] - S.loc_ptr[sub]);
        T o[K];
#pragma unroll
        for (int k = 0; k < K; ++k) o[k] = fl ? s[k] * inv : (T)0;
        stk<K, T>(S.m1 + (size_t)sub * K, o);
    }
};

// S3: reduced rhs  rhs_k + C^T D_e^-1 rhs_e  (solver.rs:360-371).  With the
// floating mean m: sum_e (C^T/D_e)[k,e] (r_e - m) = sum_e (C^T/D_e) r_e - m * rowsum_k.
template <int K, class T = double>
struct CtF {
    using Prob = SegProb;
    using Acc = T;   // sums in the storage type (FP32 in the mixed-precision inner solve)
    const SegProb* probs;
    SchwarzDevT<T> S;
    __device__ const uint32_t* seg_ptr(const Prob& p) const { return p.seg_ptr; }
    __device__ void value(const Prob&, uint32_t a, T (&v)[K]) const {
        const uint32_t e = __ldg(S.ct_col + a);
        const T f = __ldg(S.ct_val + a);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = 0.0;
        ldk<K, T>(S.rl + (size_t)e * K, v);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] *= f;
    }
    __device__ void emit(const Prob& p, uint32_t seg, const T (&s)[K]) const {
        const uint32_t row = p.seg_base + seg;
        const uint32_t slot = S.ct_row_slot[row];
        const uint32_t sub = S.slot_sub[slot];
        const uint32_t rbi = S.ct_row_red[row];
        const bool cover = S.mode[sub] == 2;
        const uint32_t nk = S.n_kept[sub];
        const T rsum = S.ct_rowsum[row];
        T m[K], rlv[K], val[K], neg[K];
        ldk<K, T>(S.m1 + (size_t)sub * K, m);
        ldk<K, T>(S.rl + (size_t)slot * K, rlv);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            val[k] = (rlv[k] - m[k]) + (s[k] - m[k] * rsum);
            neg[k] = -val[k];
        }
        stk<K, T>(S.rb + (size_t)rbi * K, val);
        if (cover) stk<K, T>(S.rb + (size_t)(rbi + nk) * K, neg);
    }
};

// S4: per-subdomain sum of the kept reduced rhs -> floating mean (m2) or the
// explicit ground's rhs (solver.rs:372-384)
template <int K, class T = double>
struct KeptSumF {
    using Prob = SegProb;
    using Acc = T;   // sums in the storage type (FP32 in the mixed-precision inner solve)
    const SegProb* probs;
    SchwarzDevT<T> S;
    __device__ const uint32_t* seg_ptr(const Prob& p) const { return p.seg_ptr; }
    __device__ void value(const Prob&, uint32_t q, T (&v)[K]) const {
        const uint32_t u = __ldg(S.ct_row_red + q);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = 0.0;
        ldk<K, T>(S.rb + (size_t)u * K, v);
    }
    __device__ void emit(const Prob& p, uint32_t seg, const T (&s)[K]) const {
        const uint32_t sub = p.seg_base + seg;
        const int m = S.mode[sub];
        T o[K];
        if (m == 0) {
            const T rn = (double)S.red_n[sub];
#pragma unroll
            for (int k = 0; k < K; ++k) o[k] = s[k] / rn;
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) o[k] = 0.0;
            if (m == 1) {
                T neg[K];
#pragma unroll
                for (int k = 0; k < K; ++k) neg[k] = -s[k];
                stk<K, T>(S.rb + (size_t)(S.red_off[sub] + S.n_kept[sub]) * K, neg);
            }
        }
        stk<K, T>(S.m2 + (size_t)sub * K, o);
    }
};

template <int K, class T = double>
__device__ __forceinline__ void reduced_rhs(const SchwarzDevT<T>& S, uint32_t u, T (&b)[K]) {
    const uint32_t s = S.red_sub[u];
    T m[K];
    ldk<K, T>(S.rb + (size_t)u * K, b);
    ldk<K, T>(S.m2 + (size_t)s * K, m);
#pragma unroll
    for (int k = 0; k < K; ++k) b[k] -= m[k];
}

// S5 (small systems): x = G b with the dense generalised inverse G
template <int K, class T = double>
struct DenseF {
    using Prob = SegProb;
    using Acc = T;   // sums in the storage type (FP32 in the mixed-precision inner solve)
    const SegProb* probs;
    SchwarzDevT<T> S;
    __device__ const uint32_t* seg_ptr(const Prob& p) const { return p.seg_ptr; }
    __device__ void value(const Prob&, uint32_t a, T (&v)[K]) const {
        T b[K];
        reduced_rhs<K, T>(S, __ldg(S.dense_col + a), b);
        const T g = __ldg(S.dense_val + a);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = g * b[k];
    }
    __device__ void emit(const Prob& p, uint32_t seg, const T (&s)[K]) const {
        const uint32_t u = S.dense_row_slot[p.seg_base + seg];
        stk<K, T>(S.xv + (size_t)u * K, s);
    }
};

// S5 (factored systems), one round of L y = b: y_u = b_u - sum_v L[u,v] y_v,
// and z_u = y_u / d_u for the backward pass.
template <int K, class T = double>
struct FwdF {
    using Prob = SegProb;
    using Acc = T;   // sums in the storage type (FP32 in the mixed-precision inner solve)
    const SegProb* probs;
    SchwarzDevT<T> S;
    __device__ const uint32_t* seg_ptr(const Prob& p) const { return p.seg_ptr; }
    __device__ void value(const Prob&, uint32_t a, T (&v)[K]) const {
        const uint32_t c = __ldg(S.fwd_col + a);
        const T l = __ldg(S.fwd_val + a);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = 0.0;
        ldk<K, T>(S.yv + (size_t)c * K, v);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] *= l;
    }
    __device__ void emit(const Prob& p, uint32_t seg, const T (&s)[K]) const {
        const uint32_t u = S.fwd_row[p.seg_base + seg];
        T b[K];
        reduced_rhs<K, T>(S, u, b);
        const T di = S.dinv[u];
        T y[K], x[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            y[k] = b[k] - s[k];
            x[k] = y[k] * di;
        }
        stk<K, T>(S.yv + (size_t)u * K, y);
        stk<K, T>(S.xv + (size_t)u * K, x);
    }
};

// dense core of a round-scheduled factor: x_core = G_core y_core, between the
// forward and the backward sweeps
template <int K, class T = double>
struct CoreF {
    using Prob = SegProb;
    using Acc = T;   // sums in the storage type (FP32 in the mixed-precision inner solve)
    const SegProb* probs;
    SchwarzDevT<T> S;
    __device__ const uint32_t* seg_ptr(const Prob& p) const { return p.seg_ptr; }
    __device__ void value(const Prob&, uint32_t a, T (&v)[K]) const {
        const uint32_t c = __ldg(S.core_col + a);
        const T g = __ldg(S.core_val + a);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = 0.0;
        ldk<K, T>(S.yv + (size_t)c * K, v);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] *= g;
    }
    __device__ void emit(const Prob& p, uint32_t seg, const T (&s)[K]) const {
        const uint32_t u = S.core_row_slot[p.seg_base + seg];
        stk<K, T>(S.xv + (size_t)u * K, s);
    }
};

// one round of L^T x = z: x_v = z_v - sum_u L[u,v] x_u (rounds in reverse)
template <int K, class T = double>
struct BwdF {
    using Prob = SegProb;
    using Acc = T;   // sums in the storage type (FP32 in the mixed-precision inner solve)
    const SegProb* probs;
    SchwarzDevT<T> S;
    __device__ const uint32_t* seg_ptr(const Prob& p) const { return p.seg_ptr; }
    __device__ void value(const Prob&, uint32_t a, T (&v)[K]) const {
        const uint32_t c = __ldg(S.bwd_col + a);
        const T l = __ldg(S.bwd_val + a);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = 0.0;
        ldk<K, T>(S.xv + (size_t)c * K, v);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] *= l;
    }
    __device__ void emit(const Prob& p, uint32_t seg, const T (&s)[K]) const {
        const uint32_t v = S.bwd_row[p.seg_base + seg];
        T x[K];
        ldk<K, T>(S.xv + (size_t)v * K, x);
#pragma unroll
        for (int k = 0; k < K; ++k) x[k] -= s[k];
        stk<K, T>(S.xv + (size_t)v * K, x);
    }
};

// S6: back-substitution  x_e = D_e^-1 rhs_e + D_e^-1 C x_k  (solver.rs:41-77);
// C is stored pre-divided by D_e, and a column with bit 31 clear reads the
// reduced solution directly (floating subdomain).
template <int K, class T = double>
struct CF {
    using Prob = SegProb;
    using Acc = T;   // sums in the storage type (FP32 in the mixed-precision inner solve)
    const SegProb* probs;
    SchwarzDevT<T> S;
    __device__ const uint32_t* seg_ptr(const Prob& p) const { return p.seg_ptr; }
    __device__ void value(const Prob&, uint32_t a, T (&v)[K]) const {
        const uint32_t cc = __ldg(S.c_col + a);
        const T c = __ldg(S.c_val + a);
        T x[K];
        if (cc & 0x80000000u) {
            kept_solution<K, T>(S, cc & 0x7fffffffu, x);
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) x[k] = 0.0;
            ldk<K, T>(S.xv + (size_t)cc * K, x);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = c * x[k];
    }
    __device__ void emit(const Prob& p, uint32_t seg, const T (&s)[K]) const {
        const uint32_t e = S.elim_slot[p.seg_base + seg];
        const uint32_t sub = S.slot_sub[e];
        const T ie = S.inv_e[e];
        T rlv[K], m[K], o[K];
        ldk<K, T>(S.rl + (size_t)e * K, rlv);
        ldk<K, T>(S.m1 + (size_t)sub * K, m);
#pragma unroll
        for (int k = 0; k < K; ++k) o[k] = (rlv[k] - m[k]) * ie + s[k];
        stk<K, T>(S.sl + (size_t)e * K, o);
    }
};

// S7: kept-block read-back and per-subdomain solution mean (floating)
template <int K, class T = double>
struct MeanF {
    using Prob = SegProb;
    using Acc = T;   // sums in the storage type (FP32 in the mixed-precision inner solve)
    const SegProb* probs;
    SchwarzDevT<T> S;
    __device__ const uint32_t* seg_ptr(const Prob& p) const { return p.seg_ptr; }
    __device__ void value(const Prob&, uint32_t j, T (&v)[K]) const {
        const uint32_t s = __ldg(S.slot_sub + j);
        const uint32_t kk = j - S.loc_ptr[s];
        const uint32_t ne = S.n_elim[s];
        if (kk < ne) {
#pragma unroll
            for (int k = 0; k < K; ++k) v[k] = 0.0;
            ldk<K, T>(S.sl + (size_t)j * K, v);
        } else {
            kept_solution<K, T>(S, S.red_off[s] + (kk - ne), v);
            stk<K, T>(S.sl + (size_t)j * K, v);
        }
    }
    __device__ void emit(const Prob& p, uint32_t seg, const T (&s)[K]) const {
        const uint32_t sub = p.seg_base + seg;
        const bool fl = S.mode[sub] == 0;
        const T inv = 1.0 / (double)(S.loc_ptr[sub + 1] - S.loc_ptr[sub]);
        T o[K];
#pragma unroll
        for (int k = 0; k < K; ++k) o[k] = fl ? s[k] * inv : (T)0;
        stk<K, T>(S.m3 + (size_t)sub * K, o);
    }
};

// S8: unfold + prolongate  z_g = sum over subdomains of w * f * (x - mean)
// (domain.rs:154-171), a gather per DOF in subdomain order.
template <int K, class T = double>
struct ProlongF {
    using Prob = SegProb;
    using Acc = T;   // sums in the storage type (FP32 in the mixed-precision inner solve)
    const SegProb* probs;
    SchwarzDevT<T> S;
    T* z;
    __device__ const uint32_t* seg_ptr(const Prob& p) const { return p.seg_ptr; }
    __device__ void value(const Prob&, uint32_t a, T (&v)[K]) const {
        const uint32_t j = __ldg(S.dof_slot + a);
        const uint32_t s = __ldg(S.slot_sub + j);
        const T sc = __ldg(S.scale + j);
        T m[K];
        ldk<K, T>(S.sl + (size_t)j * K, v);
        ldk<K, T>(S.m3 + (size_t)s * K, m);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = sc * (v[k] - m[k]);
    }
    __device__ void emit(const Prob& p, uint32_t seg, const T (&s)[K]) const {
        stk<K, T>(z + (size_t)(p.seg_base + seg) * K, s);
    }
};

// ---------------------------------------------------------------------------
// LSMR vector kernels over the DOF space

// v = d * p~ (Diagonal, operator/schwarz.rs:64-81) or v = p~ (identity)
template <int K, class T = double>
__global__ void k_diag_apply(uint32_t n, const T* __restrict__ d, const T* __restrict__ p,
                             T* __restrict__ v, const Ctl* ctl) {
    pdl_wait();
    pdl_launch_dependents();
    if (ctl && ctl->all_done) return;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const double dj = d ? (double)d[j] : 1.0;
#pragma unroll
        for (int k = 0; k < K; ++k) v[(size_t)j * K + k] = (T)(dj * (double)p[(size_t)j * K + k]);
    }
}

__device__ __forceinline__ void givens(double a, double b, double& c, double& s, double& r) {
    r = hypot(a, b);
    if (r > 0.0) {
        c = a / r;
        s = b / r;
    } else {
        c = 1.0;
        s = 0.0;
    }
}

// alpha = sqrt(<v, p~>) with the indefinite-M check (bidiag.rs:98-111), then
// one LsmrRecurrenceState::step, the SolutionState coefficients and the
// convergence test (recurrence.rs:81-255), written to the next state.
template <int K>
__global__ void __launch_bounds__(RED_THREADS)
k_alpha_step(uint32_t n, const double* __restrict__ v, const double* __restrict__ p,
             const ColState* cur, ColState* nxt, Ctl* ctl, double* partials, unsigned* counter) {
    pdl_wait();
    pdl_launch_dependents();
    if (ctl->all_done) return;
    double acc[3 * K];
#pragma unroll
    for (int i = 0; i < 3 * K; ++i) acc[i] = 0.0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double a = v[(size_t)j * K + k], b = p[(size_t)j * K + k];
            acc[3 * k] += a * b;
            acc[3 * k + 1] += a * a;
            acc[3 * k + 2] += b * b;
        }
    }
    double tot[3 * K];
    if (!grid_reduce<3 * K>(acc, partials, counter, tot) || threadIdx.x != 0) return;
    bool all = true;
    for (int k = 0; k < K; ++k) {
        ColState s = cur[k];
        if (s.done) {
            s.upd = 0;
            nxt[k] = s;
            continue;
        }
        const double beta = s.beta;
        double alpha = 0.0;
        if (beta != 0.0) {
            const double vp = tot[3 * k];
            if (vp < 0.0) {
                const double bound = sqrt(DBL_EPSILON) * sqrt(tot[3 * k + 1] * tot[3 * k + 2]);
                if (vp < -bound) {
                    s.err = 5;
                    s.done = 1;
                    s.upd = 0;
                    nxt[k] = s;
                    atomicCAS(&ctl->err, 0, 5);
                    continue;
                }
            }
            alpha = sqrt(fmax(vp, 0.0));
        }
        // ConvergenceState::observe
        s.a_norm_sq += alpha * alpha + beta * beta;
        // LsmrRecurrenceState::step
        double hc, hs, hr;
        givens(s.alpha_bar, beta, hc, hs, hr);
        const double theta_new = hs * alpha;
        const double alpha_bar_new = -hc * alpha;
        const double phi_bar_new = hs * s.phi_bar;
        const double theta_bar = s.s_bar * hr;
        double bc, bs, br;
        givens(s.c_bar * hr, theta_new, bc, bs, br);
        const double zeta = bc * s.zeta_bar;
        const double zeta_bar_new = -bs * s.zeta_bar;
        s.alpha_bar = alpha_bar_new;
        s.phi_bar = phi_bar_new;
        s.c_bar = bc;
        s.s_bar = bs;
        s.zeta_bar = zeta_bar_new;
        // SolutionState::update coefficients
        const double txd = hr * br;
        s.t_x = fabs(txd) > DBL_EPSILON ? zeta / txd : 0.0;
        const double thd = s.prev_rho * s.prev_rho_bar;
        s.t_hbar = fabs(thd) > DBL_EPSILON ? theta_bar * hr / thd : 0.0;
        s.t_h = fabs(hr) > DBL_EPSILON ? theta_new / hr : 0.0;
        s.prev_rho = hr;
        s.prev_rho_bar = br;
        // bidiagonalisation state for the next step
        s.vscale = alpha > 0.0 ? 1.0 / alpha : 1.0;
        s.alpha = alpha;
        s.beta_prev_inv = beta == 0.0 ? 0.0 : 1.0 / beta;
        s.itn += 1;
        s.upd = 1;
        // ConvergenceState::check, then the escalation rule, then the budget
        // (lsmr_from_bidiag, lsmr.rs:324-370)
        const double residual = fabs(s.phi_bar);
        if (residual <= s.abs_tol) {
            s.done = 1;
            s.stop = STOP_RESID;
        } else {
            const double an = fmax(sqrt(s.a_norm_sq), DBL_MIN);
            if (fabs(s.zeta_bar) / (an * fmax(residual, DBL_MIN)) <= s.rel_tol) {
                s.done = 1;
                s.stop = STOP_NORMAL;
            }
        }
        if (!s.done && s.stale_window > 0) {   // Staleness::should_escalate (lsmr.rs:138-152)
            const double ne = fabs(s.zeta_bar) / s.zeta0;
            if (isfinite(s.stale_prev) && s.stale_prev > 0.0) s.stale_n = ne / s.stale_prev > s.stale_thr ? s.stale_n + 1 : 0;
            s.stale_prev = ne;
            if (s.stale_n >= s.stale_window) {
                s.done = 1;
                s.stop = STOP_ESCALATED;
            }
        }
        if (!s.done && s.itn >= s.maxiter) {
            s.done = 1;
            s.stop = STOP_MAXITER;
        }
        nxt[k] = s;
        all = all && s.done;
    }
    ctl->k5_skip = 0;
    ctl->all_done = all ? 1 : 0;
}

// v <- v / alpha; h_bar, x, h update (recurrence.rs:143-191)
// Ring of the last `cap` (v, p/alpha) pairs for the windowed M-orthogonal
// reorthogonalisation (bidiag.rs:113-217, 489-512); cap = 0 disables it.
// Layout [slot][dof][K]; the e-th pair pushed (e = 0 at initialisation, the
// iteration count after each step) lives in slot e mod cap.
struct Ring {
    double* V;
    double* P;
    int cap;
};

template <int K>
__global__ void k_solution_update(uint32_t n, double* __restrict__ v, double* __restrict__ h,
                                  double* __restrict__ hb, double* __restrict__ x,
                                  const ColState* nxt, const Ctl* ctl, Ring ring = Ring{nullptr, nullptr, 0},
                                  const double* __restrict__ p = nullptr) {
    pdl_wait();
    pdl_launch_dependents();
    if (ctl->k5_skip) return;
    double vs[K], tx[K], thb[K], th[K];
    bool up[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        up[k] = nxt[k].upd != 0;
        vs[k] = nxt[k].vscale;
        tx[k] = nxt[k].t_x;
        thb[k] = nxt[k].t_hbar;
        th[k] = nxt[k].t_h;
    }
    size_t slot[K];
    double ps[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        slot[k] = ring.cap ? (size_t)(nxt[k].itn % ring.cap) : 0;
        ps[k] = nxt[k].alpha > 0.0 ? 1.0 / nxt[k].alpha : 0.0;
    }
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!up[k]) continue;
            const size_t o = (size_t)j * K + k;
            const double vn = v[o] * vs[k];
            v[o] = vn;
            const double ho = h[o];
            const double hbv = ho - thb[k] * hb[o];
            hb[o] = hbv;
            x[o] += tx[k] * hbv;
            h[o] = vn - th[k] * ho;
            if (ring.cap) {
                const size_t r = (slot[k] * n + j) * K + k;
                ring.V[r] = vn;
                ring.P[r] = p[o] * ps[k];
            }
        }
    }
}

// One step of the windowed M-orthogonalisation of v against the j-th oldest
// stored pair (bidiag.rs:489-512, modified Gram-Schmidt order): c = <v, P_e>.
// Pairs pushed so far: itn + 1; stored: the last min(itn + 1, cap).
template <int K>
__global__ void __launch_bounds__(RED_THREADS)
k_reorth_dot(uint32_t n, int j, Ring ring, const double* __restrict__ v, const ColState* cur, const Ctl* ctl,
             double* coef, double* partials, unsigned* counter) {
    pdl_wait();
    pdl_launch_dependents();
    if (ctl->all_done) return;
    size_t slot[K];
    bool ok[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const long long pushed = cur[k].itn + 1;
        const long long cnt = pushed < ring.cap ? pushed : ring.cap;
        ok[k] = !cur[k].done && j < cnt;
        slot[k] = ok[k] ? (size_t)((pushed - cnt + j) % ring.cap) : 0;
    }
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (ok[k]) acc[k] += v[(size_t)i * K + k] * ring.P[(slot[k] * n + i) * K + k];
    double tot[K];
    if (grid_reduce<K>(acc, partials, counter, tot) && threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) coef[k] = ok[k] ? tot[k] : 0.0;
}

// v -= c V_e, p -= c P_e with the coefficient of k_reorth_dot
template <int K>
__global__ void k_reorth_axpy(uint32_t n, int j, Ring ring, double* __restrict__ v, double* __restrict__ p,
                              const ColState* cur, const Ctl* ctl, const double* coef) {
    pdl_wait();
    pdl_launch_dependents();
    if (ctl->all_done) return;
    size_t slot[K];
    double c[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const long long pushed = cur[k].itn + 1;
        const long long cnt = pushed < ring.cap ? pushed : ring.cap;
        const bool ok = !cur[k].done && j < cnt;
        slot[k] = ok ? (size_t)((pushed - cnt + j) % ring.cap) : 0;
        c[k] = ok ? coef[k] : 0.0;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (c[k] == 0.0) continue;
            const size_t o = (size_t)i * K + k;
            const size_t r = (slot[k] * n + i) * K + k;
            v[o] -= c[k] * ring.V[r];
            p[o] -= c[k] * ring.P[r];
        }
}

// ---------------------------------------------------------------------------
// initialisation of a multi-RHS run (lsmr.rs:206-295, bidiag.rs:428-472)

// internal-order y and b = sqrt(w) y from column-major caller-order Y; per
// column max |b| and a non-finite flag.
template <int K>
__global__ void __launch_bounds__(RED_THREADS)
k_load_rhs(uint32_t n, uint32_t k_used, const double* __restrict__ Y, const uint32_t* __restrict__ perm,
           const double* __restrict__ sqrt_w, double* __restrict__ yint, double* __restrict__ b,
           double* partials, unsigned* counter, double* out_max, int* nonfinite) {
    pdl_wait();
    pdl_launch_dependents();
    double mx[K];
#pragma unroll
    for (int k = 0; k < K; ++k) mx[k] = 0.0;
    int bad = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t src = perm ? perm[i] : i;
        const double w = sqrt_w ? sqrt_w[i] : 1.0;
        double yv[K], bv[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double y = (uint32_t)k < k_used ? Y[(size_t)k * n + src] : 0.0;
            if (!isfinite(y)) bad = 1;
            yv[k] = y;
            bv[k] = sqrt_w ? w * y : y;
            mx[k] = fmax(mx[k], fabs(bv[k]));
        }
        // one 16-byte store per two columns of the interleaved rows
        stk<K, double>(yint + (size_t)i * K, yv);
        stk<K, double>(b + (size_t)i * K, bv);
    }
    if (bad) atomicExch(nonfinite, 1);
    // max is order independent; reuse the sum machinery on per-block maxima
    __shared__ double sm[32][K];
    __shared__ int is_last;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double m = mx[k];
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5][k] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < K; ++k) {
            double m = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, sm[w][k]);
            partials[(size_t)blockIdx.x * K + k] = m;
        }
        __threadfence();
        is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (int k = wid; k < K; k += (int)(blockDim.x >> 5)) {
            double m = 0;
            for (unsigned blk = lane; blk < gridDim.x; blk += 32) m = fmax(m, __ldcg(&partials[(size_t)blk * K + k]));
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0) out_max[k] = m;
        }
        if (threadIdx.x == 0) *counter = 0;
    }
}

// beta_1 = ||b|| (max-scaled, lsmr.rs:22-36), u = b / beta_1, and the column
// state seeded for the adjoint/preconditioner pass.
template <int K>
__global__ void __launch_bounds__(RED_THREADS)
k_norm_b(uint32_t n, const double* __restrict__ b, const double* bmax, ColState* st, double tol,
         long long maxiter, uint32_t k_used, Ctl* ctl, double* partials, unsigned* counter, int warm = 0,
         int stale_window = 0, double stale_thr = 0.0) {
    pdl_wait();
    pdl_launch_dependents();
    double acc[K];
    double sc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        acc[k] = 0.0;
        sc[k] = bmax[k] > 0.0 ? 1.0 / bmax[k] : 0.0;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double t = b[(size_t)i * K + k] * sc[k];
            acc[k] += t * t;
        }
    double tot[K];
    if (!grid_reduce<K>(acc, partials, counter, tot) || threadIdx.x != 0) return;
    // warm: b holds b - A x0; the tolerances stay relative to the original
    // ||b|| of the previous call (mlsmr, lsmr.rs:232-292), a zero residual
    // returns x0 (STOP_WARM_EXACT) and a non-finite one is an input error
    for (int k = 0; k < K; ++k) {
        const double b_orig = st[k].b_norm;
        ColState s;
        memset(&s, 0, sizeof(s));
        const double beta = bmax[k] == 0.0 ? 0.0 : bmax[k] * sqrt(tot[k]);
        s.beta = beta;
        s.b_norm = warm ? b_orig : beta;
        s.maxiter = maxiter;
        s.abs_tol = tol * s.b_norm;
        s.rel_tol = tol;
        s.stop = STOP_NONE;
        s.prev_rho = 1.0;
        s.prev_rho_bar = 1.0;
        s.beta_prev_inv = 1.0;
        s.stale_window = stale_window;
        s.stale_thr = stale_thr;
        s.stale_prev = __longlong_as_double(0x7ff8000000000000ll);   // NaN: no ratio before the first step
        if ((uint32_t)k >= k_used) {
            s.done = 1;
            s.stop = STOP_ZERO_RHS;
        } else if (warm && !isfinite(beta)) {
            s.done = 1;
            s.err = ERR_WARM_NONFINITE;
            atomicCAS(&ctl->err, 0, ERR_WARM_NONFINITE);
        } else if (beta == 0.0) {
            s.done = 1;
            s.stop = warm ? STOP_WARM_EXACT : STOP_ZERO_RHS;
        }
        st[k] = s;
    }
    ctl->all_done = 0;
    ctl->k5_skip = 0;
    ctl->bodies_left = (int)min((long long)maxiter / 2 + 2, (long long)INT_MAX);
    ctl->bodies_run = 0;
}

// Warm start (mlsmr, lsmr.rs:232-292): x0 (column-major n_dofs x k_used)
// into the interleaved layout, with a check that every entry is finite.
template <int K>
__global__ void k_load_x0(uint32_t nd, uint32_t k_used, const double* __restrict__ x0, double* __restrict__ out,
                          int* nonfinite) {
    pdl_wait();
    pdl_launch_dependents();
    int bad = 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nd; j += gridDim.x * blockDim.x) {
        double v[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            v[k] = (uint32_t)k < k_used ? x0[(size_t)k * nd + j] : 0.0;
            if (!isfinite(v[k])) bad = 1;
        }
        stk<K, double>(out + (size_t)j * K, v);
    }
    if (bad) atomicExch(nonfinite, 1);
}

// b <- b - A x0 (A = W^{1/2} D; operator apply, gather.rs:10-109) and the new
// max |b| per column for the scaled norm of k_norm_b
template <int K>
__global__ void __launch_bounds__(RED_THREADS)
k_warm_rhs(OpParams p, const double* __restrict__ x0, double* __restrict__ b, double* partials, unsigned* counter,
           double* out_max) {
    pdl_wait();
    pdl_launch_dependents();
    double mx[K];
#pragma unroll
    for (int k = 0; k < K; ++k) mx[k] = 0.0;
    const uint32_t stride = gridDim.x * blockDim.x * 4;
    for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) * 4; base < p.n; base += stride) {
        const int nr = (int)min(4u, p.n - base);
        double s[4][K];
        rows4_dx<K>(p, base, nr, x0, s);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (r >= nr) continue;
            const double w = p.sqrt_w ? p.sqrt_w[base + r] : 1.0;
            double o[K];
            ldk<K, double>(b + (size_t)(base + r) * K, o);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                o[k] -= p.sqrt_w ? w * s[r][k] : s[r][k];
                mx[k] = fmax(mx[k], fabs(o[k]));   // NaN-free unless A x0 overflowed
                if (!isfinite(o[k])) mx[k] = o[k];
            }
            stk<K, double>(b + (size_t)(base + r) * K, o);
        }
    }
    __shared__ double sm[32][K];
    __shared__ int is_last;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double m = mx[k];
        for (int o = 16; o > 0; o >>= 1) {
            const double q = __shfl_xor_sync(0xffffffffu, m, o);
            m = isfinite(m) ? (isfinite(q) ? fmax(m, q) : q) : m;
        }
        if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5][k] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < K; ++k) {
            double m = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = isfinite(m) ? (isfinite(sm[w][k]) ? fmax(m, sm[w][k]) : sm[w][k]) : m;
            partials[(size_t)blockIdx.x * K + k] = m;
        }
        __threadfence();
        is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (int k = wid; k < K; k += (int)(blockDim.x >> 5)) {
            double m = 0;
            for (unsigned blk = lane; blk < gridDim.x; blk += 32) {
                const double q = __ldcg(&partials[(size_t)blk * K + k]);
                m = isfinite(m) ? (isfinite(q) ? fmax(m, q) : q) : m;
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double q = __shfl_xor_sync(0xffffffffu, m, o);
                m = isfinite(m) ? (isfinite(q) ? fmax(m, q) : q) : m;
            }
            if (lane == 0) out_max[k] = m;
        }
        if (threadIdx.x == 0) *counter = 0;
    }
}

// x <- x + x0 after a warm-started solve (mlsmr, lsmr.rs:293-297)
template <int K>
__global__ void k_add_x0(uint32_t nd, double* __restrict__ x, const double* __restrict__ x0) {
    pdl_wait();
    pdl_launch_dependents();
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nd * K; j += gridDim.x * blockDim.x) x[j] += x0[j];
}

template <int K>
__global__ void k_scale_u(uint32_t n, const double* __restrict__ b, double* __restrict__ u,
                          const ColState* st) {
    pdl_wait();
    pdl_launch_dependents();
    double inv[K];
#pragma unroll
    for (int k = 0; k < K; ++k) inv[k] = st[k].beta > 0.0 ? 1.0 / st[k].beta : 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) u[(size_t)i * K + k] = b[(size_t)i * K + k] * inv[k];
}

// alpha_1 from <v, p~>; LsmrRecurrenceState::init (recurrence.rs:67-78)
template <int K>
__global__ void __launch_bounds__(RED_THREADS)
k_alpha_init(uint32_t n, const double* __restrict__ v, const double* __restrict__ p, ColState* st,
             ColState* st_other, Ctl* ctl, double* partials, unsigned* counter) {
    pdl_wait();
    pdl_launch_dependents();
    double acc[3 * K];
#pragma unroll
    for (int i = 0; i < 3 * K; ++i) acc[i] = 0.0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double a = v[(size_t)j * K + k], b = p[(size_t)j * K + k];
            acc[3 * k] += a * b;
            acc[3 * k + 1] += a * a;
            acc[3 * k + 2] += b * b;
        }
    double tot[3 * K];
    if (!grid_reduce<3 * K>(acc, partials, counter, tot) || threadIdx.x != 0) return;
    bool all = true;
    for (int k = 0; k < K; ++k) {
        ColState s = st[k];
        if (!s.done) {
            const double vp = tot[3 * k];
            bool bad = false;
            if (vp < 0.0) {
                const double bound = sqrt(DBL_EPSILON) * sqrt(tot[3 * k + 1] * tot[3 * k + 2]);
                bad = vp < -bound;
            }
            if (bad) {
                s.err = 5;
                s.done = 1;
                atomicCAS(&ctl->err, 0, 5);
            } else {
                const double alpha = sqrt(fmax(vp, 0.0));
                s.alpha = alpha;
                if (alpha == 0.0) {
                    s.done = 1;
                    s.stop = STOP_INIT_ZERO;
                    s.phi_bar = s.beta;  // residual_norm = rhs_norm
                } else {
                    s.vscale = 1.0 / alpha;
                    s.a_norm_sq = alpha * alpha;
                    s.alpha_bar = alpha;
                    s.phi_bar = s.beta;
                    s.c_bar = 1.0;
                    s.s_bar = 0.0;
                    s.zeta_bar = alpha * s.beta;
                    s.zeta0 = fmax(fabs(s.zeta_bar), DBL_MIN);
                    s.beta_prev_inv = 1.0;
                }
            }
        }
        s.upd = 0;
        st[k] = s;
        st_other[k] = s;
        all = all && s.done;
    }
    ctl->all_done = all ? 1 : 0;
    ctl->k5_skip = 0;
}

// v <- v / alpha_1, h = v, x = 0, h_bar = 0  (SolutionState::init)
template <int K>
__global__ void k_init_vectors(uint32_t n, double* __restrict__ v, double* __restrict__ h,
                               double* __restrict__ hb, double* __restrict__ x, const ColState* st,
                               Ring ring = Ring{nullptr, nullptr, 0}, const double* __restrict__ p = nullptr) {
    pdl_wait();
    pdl_launch_dependents();
    double vs[K], ps[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        vs[k] = (st[k].done || st[k].alpha == 0.0) ? 1.0 : st[k].vscale;
        ps[k] = st[k].alpha > 0.0 ? 1.0 / st[k].alpha : 0.0;
    }
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const size_t o = (size_t)j * K + k;
            const double vn = v[o] * vs[k];
            v[o] = vn;
            h[o] = vn;
            hb[o] = 0.0;
            x[o] = 0.0;
            if (ring.cap) {   // the first pair, slot 0
                const size_t r = (size_t)j * K + k;
                ring.V[r] = vn;
                ring.P[r] = p[o] * ps[k];
            }
        }
}

// interleaved (internal order) -> column-major caller order
template <int K>
__global__ void k_store_obs(uint32_t n, uint32_t k_used, const double* __restrict__ src,
                            const uint32_t* __restrict__ perm, double* __restrict__ dst) {
    pdl_wait();
    pdl_launch_dependents();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t d = perm ? perm[i] : i;
        double v[K];
        ldk<K, double>(src + (size_t)i * K, v);
#pragma unroll
        for (int k = 0; k < K; ++k)
            if ((uint32_t)k < k_used) dst[(size_t)k * n + d] = v[k];
    }
}
template <int K>
__global__ void k_store_dofs(uint32_t n, uint32_t k_used, const double* __restrict__ src,
                             double* __restrict__ dst) {
    pdl_wait();
    pdl_launch_dependents();
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double v[K];
        ldk<K, double>(src + (size_t)j * K, v);
#pragma unroll
        for (int k = 0; k < K; ++k)
            if ((uint32_t)k < k_used) dst[(size_t)k * n + j] = v[k];
    }
}

// ---------------------------------------------------------------------------
// Demeaning adjoint (vector-Jacobian product of z -> z - D x*(z, w)).
// With r = demeaned(z), a = v / w and s = demeaned(a) (one more solve with the
// same weights and preconditioner):  dL/dz = w * s  and
// dL/dw = -sum_columns r * (a - s).  Column-major (n, k) buffers.

__global__ void k_adjoint_rhs(uint64_t n, uint32_t k, const double* __restrict__ v,
                              const double* __restrict__ w, double* __restrict__ a) {
    pdl_wait();
    pdl_launch_dependents();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double wi = w ? w[i] : 1.0;
        for (uint32_t c = 0; c < k; ++c) a[(size_t)c * n + i] = w ? v[(size_t)c * n + i] / wi : v[(size_t)c * n + i];
    }
}

__global__ void k_demean_vjp(uint64_t n, uint32_t k, const double* __restrict__ r, const double* __restrict__ a,
                             const double* __restrict__ s, const double* __restrict__ w,
                             double* __restrict__ gz, double* __restrict__ gw) {
    pdl_wait();
    pdl_launch_dependents();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double wi = w ? w[i] : 1.0;
        double g = 0.0;
        for (uint32_t c = 0; c < k; ++c) {
            const size_t o = (size_t)c * n + i;
            const double sv = s[o];
            if (gz) gz[o] = wi * sv;
            if (gw) g -= r[o] * (a[o] - sv);
        }
        if (gw) gw[i] = g;
    }
}

}  // namespace wgpu
