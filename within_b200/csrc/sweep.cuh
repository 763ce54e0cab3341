// sweep.cuh -- the fused row sweep: one pass over the observations that does
// the gather and LSMR update u <- A v + s u (bidiag.rs:278-283) together with
// the part of the adjoint D^T (W^{1/2} u) (scatter.rs:14-73) that can be
// formed while each row's u is still in registers.
//
// Every term of the design falls into one of three classes, fixed per design
// at set-up:
//   run terms   the term's code changes rarely along the (locality-sorted) row
//               order -- the dominant sorted term, whose runs are its levels,
//               and terms such as a firm under a worker-sorted panel.  A
//               block-wide segmented scan over each 1024-row tile sums every
//               run; a run that is a whole level is written straight into A^T u,
//               other runs into a run-sum array that a later segmented
//               reduction combines per level through the level-sorted run
//               order (5x fewer entries than rows for the firm term).
//   hist terms  few coefficients (levels x columns x RHS <= 24): every thread
//               accumulates its rows into a private shared-memory histogram,
//               reduced in a fixed order per block and then over blocks.
//   other terms left to the segmented reduction over the level-sorted
//               observation permutation (segreduce.cuh).
// Runs that cross a tile boundary leave a tail partial (tile where the run
// starts) and head partials (tiles it continues into); the last CTA of the run
// adds them in tile order (one atomic counter per run, no waiting).  All sums
// have one fixed order: results are bitwise reproducible.
#pragma once
#include <cub/block/block_scan.cuh>

#include "kernels.cuh"

namespace wgpu {

constexpr int SW_THREADS = 256;
constexpr int SW_TILE = SW_THREADS * 4;   // rows per tile (4 per thread)
constexpr int SW_MAX_RUN = 3;
constexpr int SW_MAX_HIST = 2;
constexpr int SW_HIST_CAP = 24;           // histogram doubles per thread (all hist terms, all RHS)

struct SweepRun {
    int term;                   // term index in OpParams
    int direct;                 // 1: every run is a whole level (sorted term): write A^T u directly
    const uint32_t* cont_t0;    // per tile: tile where the run continuing into it starts (or UINT32_MAX)
    const uint32_t* leave_t1;   // per tile: last tile of the run leaving it (or UINT32_MAX)
    const uint32_t* leave_a;    // per tile: first row of the run leaving it
    double* run_sum;            // direct == 0: indexed by the run's first row: (row * ncol + c) * K + k
    unsigned* cnt;              // per tile completion counter of the run leaving it, kept at zero
    double* head;               // per tile partial of the run continuing into the tile: (tile*ncol + c)*K + k
    double* tail;               // per tile partial of the run leaving the tile
};

struct SweepHist {
    int term;
    int bucket0;                // first bucket: bucket = bucket0 + level * ncol + c
};

struct SweepParams {
    uint32_t n_tiles;
    int n_run, n_hist;
    SweepRun run[SW_MAX_RUN];
    SweepHist hist[SW_MAX_HIST];
    int n_buckets;              // sum over hist terms of L * ncol
    double* hist_part;          // gridDim * n_buckets * K block partials
    unsigned* hist_counter;
    double* atu;                // raw A^T u for run(direct) and hist terms: dof * K + k
};

struct SweepShared {
    cub::BlockScan<SegItem<1>, SW_THREADS>::TempStorage scan;
    int fin[2];       // start tiles of the runs this CTA completes
    double wsum[(SW_THREADS / 32) * 8];
};

// Writes the finished sum of the run that starts at `row0_run` (level `level`).
template <int K>
__device__ __forceinline__ void sweep_emit(const OpParams& p, const SweepParams& sw, const SweepRun& R,
                                           uint32_t row0_run, uint32_t level, int c, const double* v) {
    const int t = R.term;
    if (R.direct) {
        const size_t dof = (size_t)p.off[t] + (size_t)c * p.L[t] + level;
#pragma unroll
        for (int k = 0; k < K; ++k) sw.atu[dof * K + k] = v[k];
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) R.run_sum[((size_t)row0_run * p.ncol[t] + c) * K + k] = v[k];
    }
}

// One run term over one tile.  `code` are this thread's 4 row codes of the
// term, `b[r][k]` = sqrt(w) u of its rows.  A run is identified by its first
// row; the segmented scan carries the first row of the run each row belongs to
// (-1 for the run that started in an earlier tile).
template <int K>
__device__ void sweep_run_tile(const OpParams& p, const SweepParams& sw, const SweepRun& R, uint32_t tile,
                               uint32_t row0, const uint32_t (&code)[4], int nr, const double (&b)[4][K],
                               SweepShared& sh) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t t0row = tile * SW_TILE;
    const uint32_t tile_end = min(t0row + (uint32_t)SW_TILE, p.n);
    const int t = R.term;
    const int ncol = p.ncol[t];
    const uint32_t* cd = p.codes[t];
    // neighbours of this thread's rows (cached loads; no barrier)
    const uint32_t prev = (nr > 0 && row0 > 0) ? __ldg(cd + row0 - 1) : 0u;
    const uint32_t nxt = (nr > 0 && row0 + nr < p.n) ? __ldg(cd + row0 + nr) : 0u;
    int sid[4];
    bool last[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const uint32_t row = row0 + r;
        const uint32_t pc = r == 0 ? prev : code[r - 1];
        const bool head = r < nr && (row == 0 || code[r] != pc);
        // a run starts at the tile's first row only if the row is a head
        sid[r] = head ? (int)row : -1;
        const uint32_t nc = r + 1 < nr ? code[r + 1] : nxt;
        last[r] = r < nr && (row + 1 == tile_end || row + 1 == p.n || nc != code[r]);
    }
    // does the run holding the tile's last row end at the tile end?
    const bool ends_at_tile_end = tile_end >= p.n || __ldg(cd + tile_end) != __ldg(cd + tile_end - 1);
    int leaving = -1;
    for (int c = 0; c < ncol; ++c) {
        const int li = p.load[t][c];
        double val[4][K];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const double ld = (li < 0 || r >= nr) ? 1.0 : __ldg(p.loads[li] + row0 + r);
#pragma unroll
            for (int k = 0; k < K; ++k) val[r][k] = r < nr ? ld * b[r][k] : 0.0;
        }
        int sc[4] = {-1, -1, -1, -1};
#pragma unroll
        for (int k = 0; k < K; ++k) {
            SegItem<1> it[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                it[r].v[0] = val[r][k];
                it[r].sid = sid[r];
            }
            __syncthreads();   // scan storage reuse
            cub::BlockScan<SegItem<1>, SW_THREADS>(sh.scan).InclusiveScan(it, it, SegSumOp<1>());
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                val[r][k] = it[r].v[0];
                sc[r] = it[r].sid;
            }
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (!last[r]) continue;
            const bool at_end = row0 + r + 1 == tile_end;
            const int first = sc[r];
            if (first >= 0 && (!at_end || ends_at_tile_end)) {
                sweep_emit<K>(p, sw, R, (uint32_t)first, code[r], c, val[r]);
            } else if (first >= 0) {   // leaves the tile: tail partial
#pragma unroll
                for (int k = 0; k < K; ++k) R.tail[((size_t)tile * ncol + c) * K + k] = val[r][k];
                __threadfence();
                leaving = first;
            } else {                   // continues from an earlier tile: head partial
#pragma unroll
                for (int k = 0; k < K; ++k) R.head[((size_t)tile * ncol + c) * K + k] = val[r][k];
                __threadfence();
            }
        }
    }
    (void)leaving;
    (void)lane;
    (void)wid;
    __syncthreads();
    if (tid == 0) {
        // runs this tile holds a partial of: the one continuing into it and the one leaving it
        const uint32_t ids[2] = {__ldg(R.cont_t0 + tile), __ldg(R.leave_t1 + tile) == UINT32_MAX ? UINT32_MAX : tile};
        for (int j = 0; j < 2; ++j) {
            sh.fin[j] = -1;
            const uint32_t ts = ids[j];
            if (ts == UINT32_MAX) continue;
            const unsigned total = __ldg(R.leave_t1 + ts) - ts + 1;
            if (atomicAdd(&R.cnt[ts], 1u) == total - 1) sh.fin[j] = (int)ts;
        }
    }
    __syncthreads();
    for (int j = 0; j < 2; ++j) {
        const int ts = sh.fin[j];
        if (ts < 0) continue;   // uniform (shared)
        __threadfence();
        const uint32_t te = __ldg(R.leave_t1 + ts);
        for (int c = 0; c < ncol; ++c) {
            double acc[K];
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] = 0.0;
            for (uint32_t tt = (uint32_t)ts + 1 + tid; tt <= te; tt += SW_THREADS)
#pragma unroll
                for (int k = 0; k < K; ++k) acc[k] += __ldcg(&R.head[((size_t)tt * ncol + c) * K + k]);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                double v = acc[k];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if ((tid & 31) == 0) sh.wsum[(tid >> 5) * 8 + k] = v;
            }
            __syncthreads();
            if (tid == 0) {
                const uint32_t a = __ldg(R.leave_a + ts);
                const uint32_t lv = __ldg(cd + a);
                double tot[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    double v = __ldcg(&R.tail[((size_t)ts * ncol + c) * K + k]);
                    for (int w = 0; w < SW_THREADS / 32; ++w) v += sh.wsum[w * 8 + k];
                    tot[k] = v;
                }
                sweep_emit<K>(p, sw, R, a, lv, c, tot);
            }
            __syncthreads();
        }
        if (tid == 0) R.cnt[ts] = 0;
    }
}

// The sweep.  LSMR: u <- W^{1/2} D v + scale u for active columns and beta =
// ||u|| (last block); otherwise (Operator::apply_adjoint) u is read as given.
// Both: the run and hist terms' sums of W^{1/2} u, into sw.atu / run sums.
template <int K>
constexpr int sw_min_blocks() { return K >= 4 ? 2 : 4; }

template <int K, bool LSMR>
__global__ void __launch_bounds__(SW_THREADS, sw_min_blocks<K>())
k_sweep(OpParams p, SweepParams sw, const double* __restrict__ v, double* __restrict__ u, ColState* cur,
        Ctl* ctl, double* partials, unsigned* counter) {
    extern __shared__ double hist_s[];   // n_buckets * K * SW_THREADS
    __shared__ SweepShared sh;
    if (LSMR && ctl->all_done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->k5_skip = 1;
        return;
    }
    const int tid = threadIdx.x;
    const int nhb = sw.n_buckets * K;
    for (int i = tid; i < nhb * SW_THREADS; i += SW_THREADS) hist_s[i] = 0.0;
    double scale[K];
    bool act[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        act[k] = LSMR ? !cur[k].done : false;
        scale[k] = LSMR ? -(cur[k].alpha * cur[k].beta_prev_inv) : 0.0;
    }
    double accn[K];
#pragma unroll
    for (int k = 0; k < K; ++k) accn[k] = 0.0;
    __syncthreads();
    for (uint32_t tile = blockIdx.x; tile < sw.n_tiles; tile += gridDim.x) {
        const uint32_t row0 = tile * SW_TILE + tid * 4;
        const int nr = row0 < p.n ? (int)min(4u, p.n - row0) : 0;
        double b[4][K];
        if (LSMR) {
            double s[4][K];
            if (nr > 0) rows4_dx<K>(p, row0, nr, v, s);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const double w = (r < nr && p.sqrt_w) ? __ldg(p.sqrt_w + row0 + r) : 1.0;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    double nu = 0.0;
                    if (r < nr) {
                        double* up = u + (size_t)(row0 + r) * K + k;
                        nu = act[k] ? (p.sqrt_w ? w * s[r][k] : s[r][k]) + scale[k] * (*up) : *up;
                        if (act[k]) *up = nu;
                        accn[k] += nu * nu;
                    }
                    b[r][k] = p.sqrt_w ? w * nu : nu;
                }
            }
        } else {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const double w = (r < nr && p.sqrt_w) ? __ldg(p.sqrt_w + row0 + r) : 1.0;
#pragma unroll
                for (int k = 0; k < K; ++k) b[r][k] = r < nr ? w * u[(size_t)(row0 + r) * K + k] : 0.0;
            }
        }
        // hist terms: private per-thread accumulation
        for (int hh = 0; hh < sw.n_hist; ++hh) {
            const int t = sw.hist[hh].term;
            const int ncol = p.ncol[t];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (r >= nr) continue;
                const uint32_t lv = __ldg(p.codes[t] + row0 + r);
                for (int c = 0; c < ncol; ++c) {
                    const int li = p.load[t][c];
                    const double ld = li < 0 ? 1.0 : __ldg(p.loads[li] + row0 + r);
                    const int bk = sw.hist[hh].bucket0 + (int)lv * ncol + c;
#pragma unroll
                    for (int k = 0; k < K; ++k) hist_s[(size_t)(bk * K + k) * SW_THREADS + tid] += ld * b[r][k];
                }
            }
        }
        // run terms: segmented scans over the tile
        for (int j = 0; j < sw.n_run; ++j) {
            const int t = sw.run[j].term;
            uint32_t code[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) code[r] = r < nr ? __ldg(p.codes[t] + row0 + r) : 0u;
            sweep_run_tile<K>(p, sw, sw.run[j], tile, row0, code, nr, b, sh);
            __syncthreads();
        }
    }
    // block partials: ||u||^2 (LSMR) and the histogram buckets, then the last
    // block to finish adds all blocks' partials in block order.
    __syncthreads();
    const int nv = (LSMR ? K : 0) + nhb;
    for (int i = tid; i < nhb; i += SW_THREADS) {
        double a = 0.0;
        for (int q = 0; q < SW_THREADS; ++q) a += hist_s[(size_t)i * SW_THREADS + q];
        sw.hist_part[((size_t)blockIdx.x * (nhb + K)) + K + i] = a;
    }
    if (LSMR) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double vsum = warp_sum(accn[k]);
            if ((tid & 31) == 0) sh.wsum[(tid >> 5) * 8 + k] = vsum;
        }
    }
    __syncthreads();
    if (tid == 0 && LSMR) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double a = 0.0;
            for (int w = 0; w < SW_THREADS / 32; ++w) a += sh.wsum[w * 8 + k];
            sw.hist_part[(size_t)blockIdx.x * (nhb + K) + k] = a;
        }
    }
    __shared__ int is_last;
    if (tid == 0) {
        __threadfence();
        is_last = atomicAdd(sw.hist_counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    // column i of the partial table: i < K are ||u||^2 sums, then buckets
    for (int i = tid; i < nhb + K; i += SW_THREADS) {
        if (i < K && !LSMR) continue;
        double a = 0.0;
        for (unsigned blk = 0; blk < gridDim.x; ++blk) a += __ldcg(&sw.hist_part[(size_t)blk * (nhb + K) + i]);
        if (i < K) {
            if (act[i]) cur[i].beta = sqrt(a);
        } else {
            // bucket -> (hist term, level, column)
            const int bk = (i - K) / K, k = (i - K) % K;
            for (int hh = 0; hh < sw.n_hist; ++hh) {
                const int t = sw.hist[hh].term;
                const int ncol = p.ncol[t];
                const int b0 = sw.hist[hh].bucket0;
                if (bk >= b0 && bk < b0 + (int)p.L[t] * ncol) {
                    const int lv = (bk - b0) / ncol, c = (bk - b0) % ncol;
                    const size_t dof = (size_t)p.off[t] + (size_t)c * p.L[t] + lv;
                    sw.atu[dof * K + k] = a;
                }
            }
        }
    }
    if (tid == 0) *sw.hist_counter = 0;
    (void)nv;
}

// p~ <- A^T u / beta - (beta / alpha) p~ over all DOFs (bidiag.rs:474-485),
// skipping finished columns; beta == 0 (lucky breakdown) zeroes p~.
template <int K>
__global__ void k_ptilde(uint32_t nd, const double* __restrict__ atu, double* __restrict__ pt,
                         const ColState* cur, const Ctl* ctl) {
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
