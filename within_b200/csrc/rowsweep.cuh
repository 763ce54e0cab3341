// rowsweep.cuh -- the fused row sweep: one pass over the observations that
// reads each row's codes once for both directions of the design operator,
//   D v (gather.rs:10-109), the LSMR update u <- A v + s u with beta = ||u||
//   (bidiag.rs:278-283), and the part of D^T (W^{1/2} u) (scatter.rs:14-73)
//   that needs no random access to the row vectors.
//
// Work split: the rows are cut into fixed contiguous ranges, one per warp
// (grid size fixed per column count, so every sum below has one order and the
// results are bitwise reproducible).  A warp walks its range in chunks of
// 32 x R rows, lane l holding R consecutive rows.  Every term of the design is
// in one of three classes, fixed per design at set-up:
//   run terms   codes change rarely along the (locality-sorted) rows: the
//               dominant sorted term, whose runs are whole levels, and terms
//               such as a firm under a worker-sorted panel.  A warp-level
//               segmented scan (shuffles, no block barrier) sums each run, the
//               open run's partial is carried in registers from chunk to
//               chunk, and a finished run is written straight into A^T u
//               (sorted term) or into a compact run-sum array (by the run's
//               ordinal) that a segmented reduction over the level-sorted runs
//               combines afterwards.  A run that crosses a range boundary
//               leaves a tail partial (range where it starts) and head
//               partials (ranges it continues into); k_rw_fix, launched after
//               the sweep, adds them in range order.
//   hist terms  few coefficients (levels x columns <= 64): bins in shared
//               memory -- per lane when they fit (each lane adds its rows in
//               order), else per warp with each 32-row step grouped by level
//               (__match_any_sync) and summed by the group's first lane in lane
//               order; bins are then reduced over lanes, warps and blocks in
//               order.
//   rest terms  left to the segmented reduction over the level-sorted
//               observation permutation (segreduce.cuh).
// SIMPLE: every term is intercept-only (one column, no loading), chosen per
// design at set-up.
// Modes: 0 -- A^T u of a given u (Operator::apply_adjoint);  1 -- LSMR step
// (u updated and stored, beta);  2 -- normal operator A^T A p for the CG of
// the mixed-precision solve (t = A p formed in registers; stored only when
// rest terms need it);  3 -- the refinement step's FP64 residual r = b - A x,
// ||r||^2 and g = A^T r in one pass (r stored only when rest terms need it).
#pragma once
#include "pdl.cuh"
#include <type_traits>

#include "kernels.cuh"

namespace wgpu {

constexpr int RW_THREADS = 256;
constexpr int RW_WARPS = RW_THREADS / 32;
constexpr int RW_MAX_RUN = 2;
constexpr int RW_MAX_HIST = 2;
constexpr int RW_MAX_BUCKETS = 64;   // levels x columns over all hist terms
constexpr int RW_RUN_VALS = 8;       // columns x K of a run term (register carry)

template <int K>
__host__ __device__ constexpr int rw_rows() { return K >= 8 ? 2 : 4; }
template <int K>
__host__ __device__ constexpr int rw_chunk() { return 32 * rw_rows<K>(); }
template <int K>
__host__ __device__ constexpr int rw_min_blocks() { return K == 1 ? 3 : 2; }
// fixed grid: 148 SMs x resident blocks per SM
template <int K>
__host__ __device__ constexpr int rw_grid() { return 148 * rw_min_blocks<K>(); }
template <int K>
__host__ __device__ constexpr int rw_max_cols() { return RW_RUN_VALS / K < MAXC ? RW_RUN_VALS / K : MAXC; }

struct RwRun {
    int term;
    int direct;                  // runs are whole levels (sorted term): write A^T u directly
    const uint32_t* range_base;  // direct == 0: per range, ordinal of the range's first run start
    double* run_sum;             // direct == 0: [(ordinal * ncol + c) * K + k]
    double* head;                // per range: partial of the run entering the range [(g * ncol + c) * K + k]
    double* tail;                // per range: partial of the run leaving the range
};

// a run crossing range boundaries: tail of range g0 + heads of g0+1..g1
struct RwFix {
    uint32_t g0, g1;
    uint32_t id;    // direct: level; else run ordinal
    uint32_t run;   // index into RwParams::run
};

struct RwHist {
    int term;
    int bucket0;    // bucket = bucket0 + level * ncol + c
};

struct RwParams {
    uint32_t rows_per_range;     // multiple of the chunk
    int n_run, n_hist, n_buckets;
    int hist_private;            // bins per lane (buckets x K x 32 per warp), else match-grouped
    RwRun run[RW_MAX_RUN];
    RwHist hist[RW_MAX_HIST];
    const RwFix* fix;
    uint32_t n_fix;
    double* part;                // per block: [K norms | n_buckets * K bins]
    unsigned* counter;
    void* atu;                   // raw A^T u of the run(direct)/hist terms: double, or T in mode 2
};

// Shared memory of the histogram terms: per-lane bins (bytes of all warps'
// bins, 16-byte aligned) followed by one FP64 sum per bucket and warp; or
// per-warp FP64 bins plus a 32 x K staging row per warp.
template <int BIN_BYTES>
__host__ __device__ constexpr size_t rw_private_bytes(int nb) {
    return ((size_t)RW_WARPS * nb * 32 * BIN_BYTES + 15) / 16 * 16;
}
constexpr size_t RW_PRIVATE_LIMIT = 100 * 1024;   // 2 blocks per SM
// dynamic shared memory any launch can ask for: the per-lane limit, or the
// per-warp bins of RW_MAX_BUCKETS x 8 columns plus staging
constexpr size_t RW_SMEM_CAP = 104 * 1024;
static_assert(RW_SMEM_CAP >= RW_PRIVATE_LIMIT && RW_SMEM_CAP >= (size_t)RW_WARPS * (RW_MAX_BUCKETS * 8 + 32 * 8) * 8,
              "shared-memory ceiling below a reachable request");
template <int K, int BIN_BYTES>
inline size_t rw_smem_bytes(int n_buckets, int n_hist, bool& priv) {
    const int nb = n_buckets * K;
    priv = false;
    if (n_hist == 0) return 0;
    const size_t pb = rw_private_bytes<BIN_BYTES>(nb) + (size_t)RW_WARPS * nb * sizeof(double);
    if (pb <= RW_PRIVATE_LIMIT) {
        priv = true;
        return pb;
    }
    return (size_t)RW_WARPS * ((size_t)nb + 32 * K) * sizeof(double);
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <int R>
__device__ __forceinline__ void rw_load_codes(const uint32_t* __restrict__ c, uint32_t row0, int nr,
                                              uint32_t (&cd)[R]) {
    if (nr == R) {
        if constexpr (R == 8) {
            const uint4 q0 = __ldg(reinterpret_cast<const uint4*>(c + row0));
            const uint4 q1 = __ldg(reinterpret_cast<const uint4*>(c + row0 + 4));
            cd[0] = q0.x;
            cd[1] = q0.y;
            cd[2] = q0.z;
            cd[3] = q0.w;
            cd[4] = q1.x;
            cd[5] = q1.y;
            cd[6] = q1.z;
            cd[7] = q1.w;
        } else if constexpr (R == 4) {
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(c + row0));
            cd[0] = q.x;
            cd[1] = q.y;
            cd[2] = q.z;
            cd[3] = q.w;
        } else {
            const uint2 q = __ldg(reinterpret_cast<const uint2*>(c + row0));
            cd[0] = q.x;
            cd[1] = q.y;
        }
    } else {
#pragma unroll
        for (int r = 0; r < R; ++r) cd[r] = r < nr ? __ldg(c + row0 + r) : 0u;
    }
}

// N consecutive values (16-byte aligned when full) as doubles
template <int N, class T>
__device__ __forceinline__ void rw_load_vals(const T* __restrict__ src, int n_valid, double (&out)[N]) {
    if (n_valid == N) {
        if constexpr (sizeof(T) == 8) {
#pragma unroll
            for (int i = 0; i < N / 2; ++i) {
                const double2 q = *reinterpret_cast<const double2*>(src + 2 * i);
                out[2 * i] = q.x;
                out[2 * i + 1] = q.y;
            }
        } else {
#pragma unroll
            for (int i = 0; i < N / 4; ++i) {
                const float4 q = *reinterpret_cast<const float4*>(src + 4 * i);
                out[4 * i] = q.x;
                out[4 * i + 1] = q.y;
                out[4 * i + 2] = q.z;
                out[4 * i + 3] = q.w;
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) out[i] = i < n_valid ? (double)src[i] : 0.0;
    }
}

template <int N, class T>
__device__ __forceinline__ void rw_store_vals(T* __restrict__ dst, int n_valid, const T (&in)[N]) {
    if (n_valid == N) {
        if constexpr (sizeof(T) == 8) {
#pragma unroll
            for (int i = 0; i < N / 2; ++i)
                *reinterpret_cast<double2*>(dst + 2 * i) = make_double2(in[2 * i], in[2 * i + 1]);
        } else {
#pragma unroll
            for (int i = 0; i < N / 4; ++i)
                *reinterpret_cast<float4*>(dst + 4 * i) = make_float4(in[4 * i], in[4 * i + 1], in[4 * i + 2], in[4 * i + 3]);
        }
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (i < n_valid) dst[i] = in[i];
    }
}

constexpr int RW_QR = 3;   // terms whose codes stay in registers for a whole chunk

// codes of term t for the lane's rows: from the registers of the first RW_QR
// terms, else loaded
template <int R, class T>
__device__ __forceinline__ void rw_pick_codes(const OpParamsT<T>& p, int t, uint32_t row0, int nr,
                                              const uint32_t (&cdq)[RW_QR][R], uint32_t (&cd)[R]) {
    if (t < RW_QR) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            uint32_t c = cdq[0][r];
#pragma unroll
            for (int q = 1; q < RW_QR; ++q)
                if (t == q) c = cdq[q][r];
            cd[r] = c;
        }
    } else {
        rw_load_codes<R>(p.codes[t], row0, nr, cd);
    }
}

template <class T>
__device__ __forceinline__ double rw_load(const OpParamsT<T>& p, int t, int c, uint32_t row) {
    const int li = p.load[t][c];
    return li < 0 ? 1.0 : (double)__ldg(p.loads[li] + row);
}

// Block partials of ||u||^2 (modes 1, 3) and of the histogram bins in warp
// order, then in the last block to finish: grand totals in block order and
// the bins into A^T u (the runs that cross range boundaries: k_rw_fix).
template <int K, int MODE, class T, bool SIMPLE>
__device__ __forceinline__ void rw_finish(const OpParamsT<T>& p, const RwParams& rw, const double (&accn)[K],
                                          const bool (&act)[K], ColState* cur, double* sq_out, int sq_stride) {
    using TO = std::conditional_t<MODE == 2, T, double>;
    using BinT = std::conditional_t<MODE == 2, T, double>;
    constexpr bool NORM = MODE == 1 || MODE == 3;
    extern __shared__ double rw_sm[];
    __shared__ double red[RW_WARPS][K];
    __shared__ int is_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nb = rw.n_buckets * K;
    const BinT* pbins = reinterpret_cast<const BinT*>(rw_sm) + (size_t)wid * nb * 32;
    double* wsums = reinterpret_cast<double*>(reinterpret_cast<char*>(rw_sm) +
                                              rw_private_bytes<sizeof(BinT)>(nb)) + (size_t)wid * nb;
    TO* atu = reinterpret_cast<TO*>(rw.atu);
    const int stride = K + nb;
    if (rw.hist_private) {   // lanes of each warp in order
        __syncwarp();
        for (int i = lane; i < nb; i += 32) {
            double s = 0.0;
            for (int l = 0; l < 32; ++l) s += (double)pbins[i * 32 + l];
            wsums[i] = s;
        }
    }
    if (NORM) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double s = warp_sum(accn[k]);
            if (lane == 0) red[wid][k] = s;
        }
    }
    __syncthreads();
    double* mypart = rw.part + (size_t)blockIdx.x * stride;
    if (NORM && threadIdx.x < K) {
        double s = 0.0;
        for (int w = 0; w < RW_WARPS; ++w) s += red[w][threadIdx.x];
        mypart[threadIdx.x] = s;
    }
    {
        const double* base = rw.hist_private
            ? reinterpret_cast<const double*>(reinterpret_cast<const char*>(rw_sm) + rw_private_bytes<sizeof(BinT)>(nb))
            : rw_sm;
        for (int i = threadIdx.x; i < nb; i += RW_THREADS) {
            double s = 0.0;
            for (int w = 0; w < RW_WARPS; ++w) s += base[(size_t)w * nb + i];
            mypart[K + i] = s;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        is_last = atomicAdd(rw.counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    // ---- last block: grand totals in block order, bins -> A^T u
    for (int i = wid; i < stride; i += RW_WARPS) {
        if (i < K && !NORM) continue;
        const double a = warp_col_sum(rw.part, gridDim.x, stride, i);
        if (lane != 0) continue;
        if (i < K) {
            if (MODE == 1 && act[i]) cur[i].beta = sqrt(a);
            if (MODE == 3) sq_out[(size_t)i * sq_stride] = a;
            continue;
        }
        const int bk = (i - K) / K, k = (i - K) % K;
        for (int hh = 0; hh < rw.n_hist; ++hh) {
            const int t = rw.hist[hh].term;
            const int ncol = (SIMPLE ? 1 : p.ncol[t]);
            const int b0 = rw.hist[hh].bucket0;
            if (bk >= b0 && bk < b0 + (int)p.L[t] * ncol) {
                const int lv = (bk - b0) / ncol, c = (bk - b0) % ncol;
                const size_t dof = (size_t)p.off[t] + (size_t)c * p.L[t] + lv;
                atu[dof * K + k] = (TO)a;
            }
        }
    }
    if (threadIdx.x == 0) *rw.counter = 0;
}

// The runs that cross range boundaries (tail of range g0 + heads of g0+1..g1,
// in range order), one thread per run, launched after the sweep: thousands
// of short dependent load chains that would otherwise run one block's worth
// at a time at the end of the sweep.
template <int K, int MODE, class T, bool SIMPLE>
__global__ void __launch_bounds__(256)
k_rw_fix(OpParamsT<T> p, RwParams rw, const Ctl* ctl, const int* skip) {
    pdl_wait();
    pdl_launch_dependents();
    using TO = std::conditional_t<MODE == 2, T, double>;
    if (MODE == 1 && ctl->all_done) return;
    if (MODE != 1 && skip && *skip) return;
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= rw.n_fix) return;
    TO* atu = reinterpret_cast<TO*>(rw.atu);
    const RwFix fx = rw.fix[f];
    const RwRun& RR = rw.run[fx.run];
    const int t = RR.term;
    const int ncol = (SIMPLE ? 1 : p.ncol[t]);
    for (int c = 0; c < ncol; ++c)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double a = __ldcg(&RR.tail[((size_t)fx.g0 * ncol + c) * K + k]);
            for (uint32_t h = fx.g0 + 1; h <= fx.g1; ++h) a += __ldcg(&RR.head[((size_t)h * ncol + c) * K + k]);
            if (RR.direct) {
                const size_t dof = (size_t)p.off[t] + (size_t)c * p.L[t] + fx.id;
                atu[dof * K + k] = (TO)a;
            } else {
                RR.run_sum[((size_t)fx.id * ncol + c) * K + k] = a;
            }
        }
}


template <int K, int MODE, class T, bool SIMPLE>
__global__ void __launch_bounds__(RW_THREADS, rw_min_blocks<K>())
k_rowsweep(OpParamsT<T> p, RwParams rw, const T* __restrict__ v, T* __restrict__ u, ColState* cur, Ctl* ctl,
           const int* skip, int store, const T* __restrict__ rhs, double* sq_out, int sq_stride) {
    pdl_wait();
    pdl_launch_dependents();
    using TO = std::conditional_t<MODE == 2, T, double>;
    constexpr int R = rw_rows<K>();
    constexpr int CH = 32 * R;
    constexpr int MAXCR = rw_max_cols<K>();
    extern __shared__ double rw_sm[];
    if (MODE == 1 && ctl->all_done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->k5_skip = 1;
        return;
    }
    if (MODE != 1 && skip && *skip) return;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nb = rw.n_buckets * K;
    // per-lane bins hold each lane's few rows per bucket in the storage type of
    // the mode (FP32 in the FP32 normal operator); every later sum is FP64
    using BinT = std::conditional_t<MODE == 2, T, double>;
    BinT* pbins = reinterpret_cast<BinT*>(rw_sm) + (size_t)wid * nb * 32;
    double* bins = rw_sm + (size_t)wid * nb;
    double* stage = rw_sm + (size_t)RW_WARPS * nb + (size_t)wid * 32 * K;
    if (rw.hist_private) {
        for (int i = lane; i < nb * 32; i += 32) pbins[i] = (BinT)0;
    } else {
        for (int i = lane; i < nb; i += 32) bins[i] = 0.0;
    }
    __syncwarp();
    TO* atu = reinterpret_cast<TO*>(rw.atu);

    double scale[K];
    bool act[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        act[k] = MODE == 1 ? !cur[k].done : false;
        scale[k] = MODE == 1 ? -(cur[k].alpha * cur[k].beta_prev_inv) : 0.0;
    }
    double accn[K];
#pragma unroll
    for (int k = 0; k < K; ++k) accn[k] = 0.0;

    const uint32_t g = blockIdx.x * RW_WARPS + wid;
    const uint64_t r0w = (uint64_t)g * rw.rows_per_range;
    const uint32_t r0 = (uint32_t)min(r0w, (uint64_t)p.n);
    const uint32_t r1 = (uint32_t)min(r0w + rw.rows_per_range, (uint64_t)p.n);

    // warp-uniform state of the run terms
    double carry[RW_MAX_RUN][RW_RUN_VALS];
    bool foreign[RW_MAX_RUN];
    uint32_t prevc[RW_MAX_RUN];
    uint32_t heads_so_far[RW_MAX_RUN];
#pragma unroll
    for (int j = 0; j < RW_MAX_RUN; ++j) {
#pragma unroll
        for (int i = 0; i < RW_RUN_VALS; ++i) carry[j][i] = 0.0;
        foreign[j] = false;
        prevc[j] = 0u;
        heads_so_far[j] = 0u;
        if (j < rw.n_run && r0 < r1) {
            const uint32_t* cd = p.codes[rw.run[j].term];
            prevc[j] = r0 > 0 ? __ldg(cd + r0 - 1) : 0u;
            foreign[j] = r0 > 0 && __ldg(cd + r0) == prevc[j];
        }
    }

    for (uint32_t c0 = r0; c0 < r1; c0 += CH) {
        const uint32_t row0 = c0 + (uint32_t)lane * R;
        const int nr = row0 < r1 ? (int)min((uint32_t)R, r1 - row0) : 0;
        // ---- every load that depends on nothing else, issued at once: the codes
        // of the first RW_QR terms (kept for the whole chunk), u and sqrt(w)
        uint32_t cdq[RW_QR][R];
#pragma unroll
        for (int t = 0; t < RW_QR; ++t) {
            if (t < p.Q) {
                rw_load_codes<R>(p.codes[t], row0, nr, cdq[t]);
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) cdq[t][r] = 0u;
            }
        }
        double uin[R * K];
        if (MODE == 0 || MODE == 1) rw_load_vals<R * K, T>(u + (size_t)row0 * K, nr * K, uin);
        if (MODE == 3) rw_load_vals<R * K, T>(rhs + (size_t)row0 * K, nr * K, uin);
        double wv[R];
#pragma unroll
        for (int r = 0; r < R; ++r) wv[r] = (r < nr && p.sqrt_w) ? (double)__ldg(p.sqrt_w + row0 + r) : 1.0;
        // ---- row values b = W^{1/2} u (mode 0), of the updated u (mode 1), or w D p (mode 2)
        double b[R][K];
        if (MODE == 0) {
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int k = 0; k < K; ++k) b[r][k] = r < nr ? wv[r] * uin[r * K + k] : 0.0;
        } else {
            double s[R][K];
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int k = 0; k < K; ++k) s[r][k] = 0.0;
#pragma unroll
            for (int t = 0; t < RW_QR; ++t) {
                if (t >= p.Q) break;
                for (int c = 0; c < (SIMPLE ? 1 : p.ncol[t]); ++c) {
                    const size_t col = (size_t)p.off[t] + (size_t)c * p.L[t];
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        if (r >= nr) continue;
                        const double ld = (SIMPLE ? 1.0 : rw_load(p, t, c, row0 + r));
                        double xg[K];
                        ldgk<K, T>(v + (col + cdq[t][r]) * K, xg);
#pragma unroll
                        for (int k = 0; k < K; ++k) s[r][k] += xg[k] * ld;
                    }
                }
            }
            for (int t = RW_QR; t < p.Q; ++t) {
                uint32_t cd[R];
                rw_load_codes<R>(p.codes[t], row0, nr, cd);
                for (int c = 0; c < (SIMPLE ? 1 : p.ncol[t]); ++c) {
                    const size_t col = (size_t)p.off[t] + (size_t)c * p.L[t];
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        if (r >= nr) continue;
                        const double ld = (SIMPLE ? 1.0 : rw_load(p, t, c, row0 + r));
                        double xg[K];
                        ldgk<K, T>(v + (col + cd[r]) * K, xg);
#pragma unroll
                        for (int k = 0; k < K; ++k) s[r][k] += xg[k] * ld;
                    }
                }
            }
            T outv[R * K];
#pragma unroll
            for (int r = 0; r < R; ++r) {
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    double val = 0.0;
                    if (r < nr) {
                        const double av = p.sqrt_w ? wv[r] * s[r][k] : s[r][k];
                        if (MODE == 1) {
                            const double nu = act[k] ? av + scale[k] * uin[r * K + k] : uin[r * K + k];
                            const T nut = (T)nu;
                            accn[k] += (double)nut * (double)nut;
                            val = (double)nut;
                            outv[r * K + k] = nut;
                        } else if (MODE == 3) {
                            const double rr = uin[r * K + k] - av;
                            accn[k] += rr * rr;
                            val = rr;
                            outv[r * K + k] = (T)rr;
                        } else {
                            const T tt = (T)av;
                            val = (double)tt;
                            outv[r * K + k] = tt;
                        }
                    } else {
                        outv[r * K + k] = (T)0;
                    }
                    b[r][k] = p.sqrt_w ? wv[r] * val : val;
                }
            }
            // finished columns store their unchanged u back (same bytes)
            if (MODE == 1 || store) rw_store_vals<R * K, T>(u + (size_t)row0 * K, nr * K, outv);
        }

        // ---- hist terms: per-lane bins, or per-warp bins grouped by level per 32-row step
        for (int hh = 0; hh < rw.n_hist; ++hh) {
            const int t = rw.hist[hh].term;
            const int ncol = (SIMPLE ? 1 : p.ncol[t]);
            uint32_t hc[R];
            rw_pick_codes<R>(p, t, row0, nr, cdq, hc);
            if (rw.hist_private) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (r >= nr) break;
                    for (int c = 0; c < ncol; ++c) {
                        const double ld = (SIMPLE ? 1.0 : rw_load(p, t, c, row0 + r));
                        const int bk = rw.hist[hh].bucket0 + (int)hc[r] * ncol + c;
#pragma unroll
                        for (int k = 0; k < K; ++k) pbins[(bk * K + k) * 32 + lane] += (BinT)(ld * b[r][k]);
                    }
                }
                continue;
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t key = r < nr ? hc[r] : 0xffffffffu;
                const unsigned grp = __match_any_sync(FULL, key);
                const int leader = __ffs(grp) - 1;
                for (int c = 0; c < ncol; ++c) {
                    const double ld = r < nr ? (SIMPLE ? 1.0 : rw_load(p, t, c, row0 + r)) : 0.0;
#pragma unroll
                    for (int k = 0; k < K; ++k) stage[lane * K + k] = ld * b[r][k];
                    __syncwarp();
                    if (lane == leader && key != 0xffffffffu) {
                        double sum[K];
#pragma unroll
                        for (int k = 0; k < K; ++k) sum[k] = 0.0;
                        unsigned m = grp;
                        while (m) {
                            const int jl = __ffs(m) - 1;
                            m &= m - 1;
#pragma unroll
                            for (int k = 0; k < K; ++k) sum[k] += stage[jl * K + k];
                        }
                        const int bk = rw.hist[hh].bucket0 + (int)key * ncol + c;
#pragma unroll
                        for (int k = 0; k < K; ++k) bins[bk * K + k] += sum[k];
                    }
                    __syncwarp();
                }
            }
        }

        // ---- run terms: warp segmented scan with the carried open run
#pragma unroll
        for (int j = 0; j < RW_MAX_RUN; ++j) {
            if (j >= rw.n_run) break;
            const RwRun& RR = rw.run[j];
            const int t = RR.term;
            const int ncol = (SIMPLE ? 1 : p.ncol[t]);
            const uint32_t* cdp = p.codes[t];
            uint32_t cd[R];
            rw_pick_codes<R>(p, t, row0, nr, cdq, cd);
            // head flags: a row whose code differs from the previous row's
            const uint32_t upc = __shfl_up_sync(FULL, cd[R - 1], 1);
            const uint32_t pc0 = lane == 0 ? prevc[j] : upc;
            bool hd[R], en[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t pc = r == 0 ? pc0 : cd[r - 1];
                hd[r] = r < nr && (row0 + r == 0 || cd[r] != pc);
            }
            // end flags: the next row's code differs, or the data end
            const uint32_t dnc = __shfl_down_sync(FULL, cd[0], 1);
            const uint32_t nxt_row = row0 + (uint32_t)nr;
            const bool next_in_warp = lane < 31 && nr == R && row0 + R < r1;
            uint32_t nxtc = dnc;
            if (!next_in_warp && nr > 0 && nxt_row < p.n) nxtc = __ldg(cdp + nxt_row);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (r >= nr) {
                    en[r] = false;
                    continue;
                }
                if (r + 1 < nr) en[r] = cd[r + 1] != cd[r];
                else en[r] = nxt_row >= p.n || nxtc != cd[r];
            }
            // run ordinals (run terms): heads before each row within the chunk
            int before = 0, chunk_heads = 0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const unsigned hbal = __ballot_sync(FULL, hd[r]);
                before += __popc(hbal & lanemask_lt());
                chunk_heads += __popc(hbal);
            }
            const uint32_t ord_base =
                RR.direct ? 0u : __ldg(RR.range_base + g) + heads_so_far[j] + (uint32_t)before;
            const bool chunk_has_head = chunk_heads > 0;
#pragma unroll
            for (int c = 0; c < MAXCR; ++c) {
                if (c >= ncol) break;
                double val[R][K];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const double ld = r < nr ? (SIMPLE ? 1.0 : rw_load(p, t, c, row0 + r)) : 0.0;
#pragma unroll
                    for (int k = 0; k < K; ++k) val[r][k] = ld * b[r][k];
                }
                // lane aggregate: sum since the lane's last head (or the whole lane)
                bool lf = false;
                double sv[K];
#pragma unroll
                for (int k = 0; k < K; ++k) sv[k] = 0.0;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (hd[r]) {
                        lf = true;
#pragma unroll
                        for (int k = 0; k < K; ++k) sv[k] = val[r][k];
                    } else {
#pragma unroll
                        for (int k = 0; k < K; ++k) sv[k] += val[r][k];
                    }
                }
                // inclusive segmented scan over the lanes
                bool sf = lf;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    double up[K];
#pragma unroll
                    for (int k = 0; k < K; ++k) up[k] = __shfl_up_sync(FULL, sv[k], d);
                    const bool uf = __shfl_up_sync(FULL, sf ? 1 : 0, d) != 0;
                    if (lane >= d) {
                        if (!sf)
#pragma unroll
                            for (int k = 0; k < K; ++k) sv[k] += up[k];
                        sf = sf || uf;
                    }
                }
                // open run entering this lane
                double ex[K];
#pragma unroll
                for (int k = 0; k < K; ++k) ex[k] = __shfl_up_sync(FULL, sv[k], 1);
                bool exf = __shfl_up_sync(FULL, sf ? 1 : 0, 1) != 0;
                if (lane == 0) {
                    exf = false;
#pragma unroll
                    for (int k = 0; k < K; ++k) ex[k] = 0.0;
                }
                double run[K];
#pragma unroll
                for (int k = 0; k < K; ++k) run[k] = exf ? ex[k] : carry[j][c * K + k] + ex[k];
                bool lane_foreign = foreign[j] && !exf;
                uint32_t own = 0;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (r >= nr) break;
                    if (hd[r]) {
                        lane_foreign = false;
                        ++own;
#pragma unroll
                        for (int k = 0; k < K; ++k) run[k] = val[r][k];
                    } else {
#pragma unroll
                        for (int k = 0; k < K; ++k) run[k] += val[r][k];
                    }
                    if (!en[r]) continue;
                    if (lane_foreign) {   // the run started in an earlier range: head partial
#pragma unroll
                        for (int k = 0; k < K; ++k) RR.head[((size_t)g * ncol + c) * K + k] = run[k];
                    } else if (RR.direct) {
                        const size_t dof = (size_t)p.off[t] + (size_t)c * p.L[t] + cd[r];
#pragma unroll
                        for (int k = 0; k < K; ++k) atu[dof * K + k] = (TO)run[k];
                    } else {
                        const size_t ord = (size_t)(ord_base + own - 1);
#pragma unroll
                        for (int k = 0; k < K; ++k) RR.run_sum[(ord * ncol + c) * K + k] = run[k];
                    }
                }
                // carry the open run into the next chunk
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const double incl = __shfl_sync(FULL, sv[k], 31);
                    carry[j][c * K + k] = chunk_has_head ? incl : carry[j][c * K + k] + incl;
                }
            }
            foreign[j] = foreign[j] && !chunk_has_head;
            heads_so_far[j] += (uint32_t)chunk_heads;
            prevc[j] = __shfl_sync(FULL, cd[R - 1], 31);
        }
    }
    // ---- range end: the open run's partial -- the tail of a run that started
    // in this range, or (no run start in the range) the head partial of a run
    // that continues past the range; a run ending exactly at the range end was
    // written above.
    if (r0 < r1 && lane == 0) {
#pragma unroll
        for (int j = 0; j < RW_MAX_RUN; ++j) {
            if (j >= rw.n_run) break;
            const RwRun& RR = rw.run[j];
            const int ncol = (SIMPLE ? 1 : p.ncol[RR.term]);
            const uint32_t* cdp = p.codes[RR.term];
            const bool cont = r1 < p.n && __ldg(cdp + r1) == __ldg(cdp + r1 - 1);
            if (foreign[j] && !cont) continue;
            double* dst = foreign[j] ? RR.head : RR.tail;
#pragma unroll
            for (int c = 0; c < MAXCR; ++c) {
                if (c >= ncol) break;
#pragma unroll
                for (int k = 0; k < K; ++k) dst[((size_t)g * ncol + c) * K + k] = carry[j][c * K + k];
            }
        }
    }

    rw_finish<K, MODE, T, SIMPLE>(p, rw, accn, act, cur, sq_out, sq_stride);
}

// p~ <- A^T u / beta - (beta / alpha) p~ over all DOFs (bidiag.rs:474-485),
// skipping finished columns; beta == 0 (lucky breakdown) zeroes p~.
template <int K>
__global__ void k_ptilde(uint32_t nd, const double* __restrict__ atu, double* __restrict__ pt,
                         const ColState* cur, const Ctl* ctl) {
    pdl_wait();
    pdl_launch_dependents();
    if (ctl->all_done) return;
    double inv[K], coef[K];
    bool act[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        act[k] = !cur[k].done;
        const double beta = cur[k].beta;
        inv[k] = beta == 0.0 ? 0.0 : 1.0 / beta;
        coef[k] = beta == 0.0 ? 0.0 : beta / cur[k].alpha;
    }
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nd; j += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (act[k]) {
                const size_t o = (size_t)j * K + k;
                pt[o] = atu[o] * inv[k] - coef[k] * pt[o];
            }
}

}  // namespace wgpu
