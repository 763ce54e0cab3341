// tsweep.cuh -- the staged row sweep: the fused row sweep of rowsweep.cuh for
// intercept-only designs of at most three terms, with the observation
// streams (codes of every term, the row vector u, sqrt(w)) brought into
// shared memory by the TMA engine ahead of use.
//
// Same work split, run bookkeeping and outputs as k_rowsweep (one contiguous
// warp range per warp; run sums straight into A^T u for the sorted term or
// into the run-sum array by ordinal; per-lane histogram bins; head and tail
// partials of the runs that cross range boundaries, added by k_rw_fix; the
// block partials and bins finished by rw_finish), so the host plan and the
// launches around it are shared.  What differs:
//  - every warp owns a ring of TS_STAGES chunk buffers in shared memory;
//    lane 0 issues one cp.async.bulk per stream and chunk TS_STAGES - 1 chunks
//    ahead of the one being processed, completing on the stage's mbarrier,
//    so HBM streams while the warp gathers coefficients and scans runs and no
//    register holds a load in flight;
//  - the term classes are compile-time: NRUN run terms and NHIST histogram
//    terms (their term indices are runtime, warp-uniform), every loop over
//    terms, rows and columns unrolled;
//  - a run is emitted when the next run's head is seen (or at the range end),
//    so no look-ahead load of the next chunk's first code is needed; the
//    lane segmented scan uses the ballot of lane heads instead of shuffled
//    flags.
// A term's codes are summed into A v in term order, as in k_rowsweep, so both
// sweeps give the same u bit for bit.
#pragma once
#include "pdl.cuh"

#include "bulk.cuh"
#include "rowsweep.cuh"

namespace wgpu {

constexpr int TS_STAGES = 3;
constexpr int TS_BLOCKS_PER_SM = 2;
constexpr int TS_GRID = 148 * TS_BLOCKS_PER_SM;
constexpr int TS_MAXQ = 3;

// Bytes of one chunk buffer: codes of NQ terms, u (K columns), sqrt(w).
template <int K>
__host__ __device__ constexpr uint32_t ts_chunk_bytes(int nq, bool weighted) {
    return (uint32_t)(rw_chunk<K>() * (4 * nq + 8 * K + (weighted ? 8 : 0)));
}

// Dynamic shared memory: the histogram area rw_finish reads (per-lane bins,
// then one FP64 sum per bucket and warp), the rings, then the barriers.
template <int K>
__host__ __device__ constexpr size_t ts_hist_bytes(int n_buckets, int n_hist) {
    return n_hist == 0 ? 0
                       : rw_private_bytes<8>(n_buckets * K) + (size_t)RW_WARPS * n_buckets * K * sizeof(double);
}
template <int K>
__host__ __device__ constexpr size_t ts_ring_offset(int n_buckets, int n_hist) {
    return (ts_hist_bytes<K>(n_buckets, n_hist) + 127) / 128 * 128;
}
template <int K>
__host__ __device__ constexpr size_t ts_smem_bytes(int n_buckets, int n_hist, int nq, bool weighted) {
    return ts_ring_offset<K>(n_buckets, n_hist) + (size_t)RW_WARPS * TS_STAGES * ts_chunk_bytes<K>(nq, weighted) +
           (size_t)RW_WARPS * TS_STAGES * sizeof(uint64_t);
}
constexpr size_t TS_SMEM_CAP = 112 * 1024;   // two blocks per SM

struct TsSlots {
    int term[TS_MAXQ];   // slot -> term: the run terms (rw.run order), then the hist terms, then the rest
};

// ring geometry of one warp
template <int K, int NQ, bool WTD>
struct TsRing {
    static constexpr int CH = rw_chunk<K>();
    static constexpr uint32_t CODE_B = CH * 4;
    static constexpr uint32_t U_B = CH * K * 8;
    static constexpr uint32_t W_B = WTD ? CH * 8 : 0;
    static constexpr uint32_t STAGE_B = NQ * CODE_B + U_B + W_B;
};

// lane 0: issue the bulk copies of chunk c0 (rows [c0, c0 + rows), rows a
// multiple of 4 so every size is a multiple of 16 bytes) into stage `st`
template <int K, int NQ, bool WTD, class T>
__device__ __forceinline__ void ts_issue(char* stage, uint64_t* bar, const OpParamsT<T>& p, const T* u,
                                         uint32_t c0, uint32_t rows) {
    using RG = TsRing<K, NQ, WTD>;
    const uint32_t code_b = rows * 4, u_b = rows * K * 8, w_b = WTD ? rows * 8 : 0;
    mbar_arrive_expect_tx(bar, NQ * code_b + u_b + w_b);
    if (rows == 0) return;
#pragma unroll
    for (int t = 0; t < NQ; ++t) bulk_g2s(stage + t * RG::CODE_B, p.codes[t] + c0, code_b, bar);
    bulk_g2s(stage + NQ * RG::CODE_B, u + (size_t)c0 * K, u_b, bar);
    if constexpr (WTD) bulk_g2s(stage + NQ * RG::CODE_B + RG::U_B, p.sqrt_w + c0, w_b, bar);
}

template <int K, int MODE, int NQ, int NRUN, int NHIST, bool WTD>
__global__ void __launch_bounds__(RW_THREADS, TS_BLOCKS_PER_SM)
k_tsweep(OpParams p, RwParams rw, TsSlots sl, const double* __restrict__ v, double* __restrict__ u,
         ColState* cur, Ctl* ctl, int* err) {
    pdl_wait();
    pdl_launch_dependents();
    static_assert(NQ >= 1 && NQ <= TS_MAXQ && NRUN >= 1 && NRUN <= RW_MAX_RUN && NHIST <= RW_MAX_HIST &&
                      NRUN + NHIST <= NQ,
                  "staged sweep: unsupported term classes");
    constexpr int R = rw_rows<K>();
    constexpr int CH = 32 * R;
    using RG = TsRing<K, NQ, WTD>;
    extern __shared__ double rw_sm[];
    if (MODE == 1 && ctl->all_done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->k5_skip = 1;
        return;
    }
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nb = rw.n_buckets * K;
    double* pbins = rw_sm + (size_t)wid * nb * 32;
    if (NHIST > 0)
        for (int i = lane; i < nb * 32; i += 32) pbins[i] = 0.0;
    char* ring = reinterpret_cast<char*>(rw_sm) + ts_ring_offset<K>(rw.n_buckets, NHIST) +
                 (size_t)wid * TS_STAGES * RG::STAGE_B;
    uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(rw_sm) +
                                                 ts_ring_offset<K>(rw.n_buckets, NHIST) +
                                                 (size_t)RW_WARPS * TS_STAGES * RG::STAGE_B) +
                     wid * TS_STAGES;

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
    const uint32_t n_chunks = (r1 - r0 + CH - 1) / CH;

    // slot terms (warp-uniform)
    int st_run[NRUN], st_hist[NHIST > 0 ? NHIST : 1];
#pragma unroll
    for (int j = 0; j < NRUN; ++j) st_run[j] = sl.term[j];
#pragma unroll
    for (int h = 0; h < NHIST; ++h) st_hist[h] = sl.term[NRUN + h];

    // run-term state (warp-uniform except the carry, which every lane holds)
    double carry[NRUN][K];
    bool started[NRUN];      // the open run's head lies in this range
    uint32_t prevc[NRUN];    // code of the row before the chunk
    uint32_t heads[NRUN];    // heads seen in the range before the chunk
#pragma unroll
    for (int j = 0; j < NRUN; ++j) {
#pragma unroll
        for (int k = 0; k < K; ++k) carry[j][k] = 0.0;
        started[j] = false;
        heads[j] = 0;
        prevc[j] = 0u;
        if (r0 < r1 && r0 > 0) prevc[j] = __ldg(p.codes[st_run[j]] + r0 - 1);
    }

    // ring set-up and prologue (lane 0 issues, the warp waits)
    if (lane == 0) {
        for (int s = 0; s < TS_STAGES; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
    }
    __syncwarp();
    auto bulk_rows = [&](uint32_t j) -> uint32_t {
        const uint32_t c0 = r0 + j * CH;
        return min((uint32_t)CH, r1 - c0) & ~3u;
    };
    if (lane == 0)
        for (uint32_t j = 0; j < (uint32_t)TS_STAGES && j < n_chunks; ++j)
            ts_issue<K, NQ, WTD, double>(ring + j * RG::STAGE_B, &bars[j], p, u, r0 + j * CH, bulk_rows(j));
    bool failed = false;
    uint32_t failed_at = 0;

    for (uint32_t j = 0; j < n_chunks; ++j) {
        const int stg = (int)(j % TS_STAGES);
        const uint32_t par = (j / TS_STAGES) & 1u;
        const bool landed = mbar_wait_bounded(&bars[stg], par);
        if (!__all_sync(FULL, landed)) {   // warp-uniform: every lane leaves together
            failed = true;
            failed_at = j;
            break;
        }
        const char* sp = ring + stg * RG::STAGE_B;
        const uint32_t c0 = r0 + j * CH;
        const uint32_t nbulk = bulk_rows(j);
        const uint32_t row0 = c0 + (uint32_t)lane * R;
        const int nr = row0 < r1 ? (int)min((uint32_t)R, r1 - row0) : 0;
        const bool in_smem = row0 + R <= c0 + nbulk;   // this lane's rows were copied
        // ---- this lane's rows: codes of every term, u (K columns), sqrt(w)
        uint32_t cd[NQ][R];
        double uin[R * K];
        double wv[R];
        if (in_smem) {
#pragma unroll
            for (int t = 0; t < NQ; ++t) {
                const uint32_t* sc = reinterpret_cast<const uint32_t*>(sp + t * RG::CODE_B) + lane * R;
                if constexpr (R == 4) {
                    const uint4 q = *reinterpret_cast<const uint4*>(sc);
                    cd[t][0] = q.x;
                    cd[t][1] = q.y;
                    cd[t][2] = q.z;
                    cd[t][3] = q.w;
                } else {
                    const uint2 q = *reinterpret_cast<const uint2*>(sc);
                    cd[t][0] = q.x;
                    cd[t][1] = q.y;
                }
            }
            const double* su = reinterpret_cast<const double*>(sp + NQ * RG::CODE_B) + lane * R * K;
#pragma unroll
            for (int i = 0; i < R * K / 2; ++i) {
                const double2 q = reinterpret_cast<const double2*>(su)[i];
                uin[2 * i] = q.x;
                uin[2 * i + 1] = q.y;
            }
            if constexpr (WTD) {
                const double* sw = reinterpret_cast<const double*>(sp + NQ * RG::CODE_B + RG::U_B) + lane * R;
#pragma unroll
                for (int r = 0; r < R; ++r) wv[r] = sw[r];
            }
        } else {   // the ragged end of the data: plain loads
#pragma unroll
            for (int t = 0; t < NQ; ++t)
#pragma unroll
                for (int r = 0; r < R; ++r) cd[t][r] = r < nr ? __ldg(p.codes[t] + row0 + r) : 0u;
#pragma unroll
            for (int i = 0; i < R * K; ++i) uin[i] = i < nr * K ? u[(size_t)row0 * K + i] : 0.0;
            if constexpr (WTD) {
#pragma unroll
                for (int r = 0; r < R; ++r) wv[r] = r < nr ? __ldg(p.sqrt_w + row0 + r) : 0.0;
            }
        }
        if constexpr (!WTD) {
#pragma unroll
            for (int r = 0; r < R; ++r) wv[r] = 1.0;
        }
        __syncwarp();
        // every lane has its rows in registers: the stage refills with chunk j + TS_STAGES
        if (lane == 0 && j + TS_STAGES < n_chunks) {
            fence_proxy_async_smem();
            ts_issue<K, NQ, WTD, double>(ring + stg * RG::STAGE_B, &bars[stg], p, u, c0 + TS_STAGES * CH,
                                         bulk_rows(j + TS_STAGES));
        }

        // ---- row values b = W^{1/2} u (mode 0) or of the updated u (mode 1)
        double b[R][K];
        if constexpr (MODE == 0) {
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
            for (int t = 0; t < NQ; ++t) {
                const size_t col = p.off[t];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (r >= nr) continue;
                    double xg[K];
                    ldgk<K, double>(v + (col + cd[t][r]) * K, xg);
#pragma unroll
                    for (int k = 0; k < K; ++k) s[r][k] += xg[k];
                }
            }
            double outv[R * K];
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    double val = 0.0;
                    if (r < nr) {
                        const double av = WTD ? wv[r] * s[r][k] : s[r][k];
                        val = act[k] ? av + scale[k] * uin[r * K + k] : uin[r * K + k];
                        accn[k] += val * val;
                    }
                    outv[r * K + k] = val;
                    b[r][k] = WTD ? wv[r] * val : val;
                }
            if (in_smem) {
                double* dst = u + (size_t)row0 * K;
#pragma unroll
                for (int i = 0; i < R * K / 2; ++i)
                    reinterpret_cast<double2*>(dst)[i] = make_double2(outv[2 * i], outv[2 * i + 1]);
            } else {
#pragma unroll
                for (int i = 0; i < R * K; ++i)
                    if (i < nr * K) u[(size_t)row0 * K + i] = outv[i];
            }
        }

        // ---- hist terms: per-lane bins, each lane adds its rows in order
#pragma unroll
        for (int h = 0; h < NHIST; ++h) {
            const int t = st_hist[h];
            const int b0 = rw.hist[h].bucket0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (r >= nr) continue;
                uint32_t c = cd[0][r];
#pragma unroll
                for (int q = 1; q < NQ; ++q)
                    if (t == q) c = cd[q][r];
                const int bk = b0 + (int)c;
#pragma unroll
                for (int k = 0; k < K; ++k) pbins[(bk * K + k) * 32 + lane] += b[r][k];
            }
        }

        // ---- run terms
#pragma unroll
        for (int jr = 0; jr < NRUN; ++jr) {
            const int t = st_run[jr];
            const RwRun& RR = rw.run[jr];
            uint32_t c[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                uint32_t x = cd[0][r];
#pragma unroll
                for (int q = 1; q < NQ; ++q)
                    if (t == q) x = cd[q][r];
                c[r] = x;
            }
            const uint32_t upc = __shfl_up_sync(FULL, c[R - 1], 1);
            const uint32_t pc0 = lane == 0 ? prevc[jr] : upc;
            bool hd[R];
            int lane_heads = 0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t pc = r == 0 ? pc0 : c[r - 1];
                hd[r] = r < nr && (row0 + r == 0 || c[r] != pc);
                lane_heads += hd[r] ? 1 : 0;
            }
            // lane aggregate: sum since the lane's last head (or of the whole lane)
            double sv[K];
#pragma unroll
            for (int k = 0; k < K; ++k) sv[k] = 0.0;
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int k = 0; k < K; ++k) sv[k] = hd[r] ? b[r][k] : sv[k] + b[r][k];
            const unsigned hm = __ballot_sync(FULL, lane_heads > 0);
            const unsigned lt = lanemask_lt();
            const int hl = 31 - __clz(hm & (lt | (1u << lane)));   // last lane <= lane with a head, or -1
            const int hl0 = hl < 0 ? 0 : hl;
            // segmented inclusive scan over the lanes
#pragma unroll
            for (int d = 1; d < 32; d <<= 1)
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const double up = __shfl_up_sync(FULL, sv[k], d);
                    if (lane - d >= hl0) sv[k] += up;
                }
            // the run open at the start of this lane's rows
            const bool exf = (hm & lt) != 0;
            double run[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                double ex = __shfl_up_sync(FULL, sv[k], 1);
                if (lane == 0) ex = 0.0;
                run[k] = exf ? ex : carry[jr][k] + ex;
            }
            bool in_range = exf || started[jr];
            // heads before this lane within the chunk (ordinals of the runs of a non-direct term)
            // (the chunk's head count only matters to a term summed by run ordinal)
            uint32_t ord = 0, chunk_heads = 0;
            if (!RR.direct) {
                int before = 0;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const unsigned bl = __ballot_sync(FULL, hd[r]);
                    before += __popc(bl & lt);
                    chunk_heads += (uint32_t)__popc(bl);
                }
                ord = __ldg(RR.range_base + g) + heads[jr] + (uint32_t)before;   // ordinal of the next head
            }
            // a head ends the run before it: a complete run (its head lies in this
            // range), or the head partial of a run that started in an earlier range
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (hd[r]) {
                    if (row0 + r > r0) {
                        if (!in_range) {
#pragma unroll
                            for (int k = 0; k < K; ++k) RR.head[(size_t)g * K + k] = run[k];
                        } else if (RR.direct) {
                            const uint32_t lvl = r == 0 ? pc0 : c[r - 1];
                            const size_t dof = (size_t)p.off[t] + lvl;
#pragma unroll
                            for (int k = 0; k < K; ++k) reinterpret_cast<double*>(rw.atu)[dof * K + k] = run[k];
                        } else {
#pragma unroll
                            for (int k = 0; k < K; ++k) RR.run_sum[(size_t)(ord - 1) * K + k] = run[k];
                        }
                    }
                    ++ord;
                    in_range = true;
#pragma unroll
                    for (int k = 0; k < K; ++k) run[k] = b[r][k];
                } else {
#pragma unroll
                    for (int k = 0; k < K; ++k) run[k] += b[r][k];
                }
            }
            // carry the open run into the next chunk
            const bool chunk_has_head = hm != 0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const double incl = __shfl_sync(FULL, sv[k], 31);
                carry[jr][k] = chunk_has_head ? incl : carry[jr][k] + incl;
            }
            started[jr] = started[jr] || chunk_has_head;
            heads[jr] += chunk_heads;
            prevc[jr] = __shfl_sync(FULL, c[R - 1], 31);
        }
    }

    if (failed) {
        // a copy did not land in time: record it, then wait (bounded) for the
        // copies this warp still has in flight before leaving
        if (lane == 0) atomicExch(err, ERR_WAIT_TIMEOUT);
        for (uint32_t jj = failed_at; jj < n_chunks && jj < failed_at + TS_STAGES; ++jj)
            (void)mbar_wait_bounded(&bars[jj % TS_STAGES], (jj / TS_STAGES) & 1u);
    }

    // ---- range end: the open run -- complete when it ends exactly at the range end
    // and started here, else the tail (started here, continues) or the head
    // partial (started earlier)
    if (!failed && r0 < r1 && lane == 0) {
#pragma unroll
        for (int jr = 0; jr < NRUN; ++jr) {
            const RwRun& RR = rw.run[jr];
            const int t = st_run[jr];
            const uint32_t* cdp = p.codes[t];
            const uint32_t last = __ldg(cdp + r1 - 1);
            const bool cont = r1 < p.n && __ldg(cdp + r1) == last;
            double* dst;
            size_t idx;
            if (!started[jr]) {
                dst = RR.head;
                idx = g;
            } else if (cont) {
                dst = RR.tail;
                idx = g;
            } else if (RR.direct) {
                dst = reinterpret_cast<double*>(rw.atu);
                idx = (size_t)p.off[t] + last;
            } else {
                dst = RR.run_sum;
                idx = (size_t)__ldg(RR.range_base + g) + heads[jr] - 1;
            }
#pragma unroll
            for (int k = 0; k < K; ++k) dst[idx * K + k] = carry[jr][k];
        }
    }

    rw_finish<K, MODE, double, true>(p, rw, accn, act, cur, nullptr, 0);
}

}  // namespace wgpu

namespace wgpu {

// ---------------------------------------------------------------------------
// Staged gather y = W^{1/2} D x (Operator::apply, gather.rs:10-109) and
// demeaning out = yint - D x (solver.rs:468-473) for intercept-only designs
// of at most three terms, one column: every warp walks chunks of 128 rows
// (chunk w, w + warps, ...), its codes (and yint, sqrt(w)) brought into a
// per-warp shared-memory ring by bulk copies TS_STAGES - 1 chunks ahead; the
// terms are summed in term order as in k_apply / k_demean (same bits).
constexpr int TG_BLOCKS_PER_SM = 3;
constexpr int TG_GRID = 148 * TG_BLOCKS_PER_SM;
constexpr int TG_CH = 128;

template <int NQ, bool WTD, bool DEMEAN>
struct TgRing {
    static constexpr uint32_t CODE_B = TG_CH * 4;
    static constexpr uint32_t Y_B = DEMEAN ? TG_CH * 8 : 0;
    static constexpr uint32_t W_B = WTD ? TG_CH * 8 : 0;
    static constexpr uint32_t STAGE_B = NQ * CODE_B + Y_B + W_B;
};
template <int NQ, bool WTD, bool DEMEAN>
__host__ __device__ constexpr size_t tg_smem_bytes() {
    return (size_t)RW_WARPS * TS_STAGES * (TgRing<NQ, WTD, DEMEAN>::STAGE_B + sizeof(uint64_t));
}

template <int NQ, bool WTD, bool DEMEAN>
__device__ __forceinline__ void tg_issue(char* stage, uint64_t* bar, const OpParams& p, const double* yint,
                                         uint32_t c0, uint32_t rows) {
    using RG = TgRing<NQ, WTD, DEMEAN>;
    mbar_arrive_expect_tx(bar, rows * (4 * NQ + (DEMEAN ? 8 : 0) + (WTD ? 8 : 0)));
    if (rows == 0) return;
#pragma unroll
    for (int t = 0; t < NQ; ++t) bulk_g2s(stage + t * RG::CODE_B, p.codes[t] + c0, rows * 4, bar);
    if constexpr (DEMEAN) bulk_g2s(stage + NQ * RG::CODE_B, yint + c0, rows * 8, bar);
    if constexpr (WTD) bulk_g2s(stage + NQ * RG::CODE_B + RG::Y_B, p.sqrt_w + c0, rows * 8, bar);
}

template <int NQ, bool WTD, bool DEMEAN>
__global__ void __launch_bounds__(RW_THREADS, TG_BLOCKS_PER_SM)
k_tgather(OpParams p, const double* __restrict__ x, const double* __restrict__ yint, double* __restrict__ out,
          const int* skip, int* err) {
    pdl_wait();
    pdl_launch_dependents();
    using RG = TgRing<NQ, WTD, DEMEAN>;
    constexpr int R = 4;
    extern __shared__ __align__(128) unsigned char tg_sm[];
    if (skip && *skip) return;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    char* ring = reinterpret_cast<char*>(tg_sm) + (size_t)wid * TS_STAGES * RG::STAGE_B;
    uint64_t* bars = reinterpret_cast<uint64_t*>(tg_sm + (size_t)RW_WARPS * TS_STAGES * RG::STAGE_B) +
                     wid * TS_STAGES;
    const uint32_t warps = gridDim.x * RW_WARPS;
    const uint32_t w0 = blockIdx.x * RW_WARPS + wid;
    const uint32_t n_total = (p.n + TG_CH - 1) / TG_CH;
    const uint32_t n_mine = w0 < n_total ? (n_total - w0 + warps - 1) / warps : 0;   // chunks w0, w0 + warps, ...
    auto chunk0 = [&](uint32_t j) -> uint32_t { return (w0 + j * warps) * TG_CH; };
    auto bulk_rows = [&](uint32_t j) -> uint32_t { return min((uint32_t)TG_CH, p.n - chunk0(j)) & ~3u; };
    if (lane == 0) {
        for (int s = 0; s < TS_STAGES; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
    }
    __syncwarp();
    if (lane == 0)
        for (uint32_t j = 0; j < (uint32_t)TS_STAGES && j < n_mine; ++j)
            tg_issue<NQ, WTD, DEMEAN>(ring + j * RG::STAGE_B, &bars[j], p, yint, chunk0(j), bulk_rows(j));
    bool failed = false;
    uint32_t failed_at = 0;
    for (uint32_t j = 0; j < n_mine; ++j) {
        const int stg = (int)(j % TS_STAGES);
        const bool landed = mbar_wait_bounded(&bars[stg], (j / TS_STAGES) & 1u);
        if (!__all_sync(FULL, landed)) {
            failed = true;
            failed_at = j;
            break;
        }
        const char* sp = ring + stg * RG::STAGE_B;
        const uint32_t c0 = chunk0(j);
        const uint32_t nbulk = bulk_rows(j);
        const uint32_t row0 = c0 + (uint32_t)lane * R;
        const int nr = row0 < p.n ? (int)min((uint32_t)R, p.n - row0) : 0;
        const bool in_smem = row0 + R <= c0 + nbulk;
        uint32_t cd[NQ][R];
        double yv[R], wv[R];
        if (in_smem) {
#pragma unroll
            for (int t = 0; t < NQ; ++t) {
                const uint4 q = reinterpret_cast<const uint4*>(sp + t * RG::CODE_B)[lane];
                cd[t][0] = q.x;
                cd[t][1] = q.y;
                cd[t][2] = q.z;
                cd[t][3] = q.w;
            }
            if constexpr (DEMEAN) {
                const double2* sy = reinterpret_cast<const double2*>(sp + NQ * RG::CODE_B) + lane * 2;
                const double2 a = sy[0], b = sy[1];
                yv[0] = a.x;
                yv[1] = a.y;
                yv[2] = b.x;
                yv[3] = b.y;
            }
            if constexpr (WTD) {
                const double2* sw = reinterpret_cast<const double2*>(sp + NQ * RG::CODE_B + RG::Y_B) + lane * 2;
                const double2 a = sw[0], b = sw[1];
                wv[0] = a.x;
                wv[1] = a.y;
                wv[2] = b.x;
                wv[3] = b.y;
            }
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) {
#pragma unroll
                for (int t = 0; t < NQ; ++t) cd[t][r] = r < nr ? __ldg(p.codes[t] + row0 + r) : 0u;
                if constexpr (DEMEAN) yv[r] = r < nr ? yint[row0 + r] : 0.0;
                if constexpr (WTD) wv[r] = r < nr ? __ldg(p.sqrt_w + row0 + r) : 0.0;
            }
        }
        __syncwarp();
        if (lane == 0 && j + TS_STAGES < n_mine) {
            fence_proxy_async_smem();
            tg_issue<NQ, WTD, DEMEAN>(ring + stg * RG::STAGE_B, &bars[stg], p, yint, chunk0(j + TS_STAGES),
                                      bulk_rows(j + TS_STAGES));
        }
        double s[R];
#pragma unroll
        for (int r = 0; r < R; ++r) s[r] = 0.0;
#pragma unroll
        for (int t = 0; t < NQ; ++t)
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (r < nr) s[r] += __ldg(x + (size_t)p.off[t] + cd[t][r]);
        double o[R];
#pragma unroll
        for (int r = 0; r < R; ++r) o[r] = DEMEAN ? yv[r] - s[r] : (WTD ? wv[r] * s[r] : s[r]);
        if (in_smem) {
            double2* dst = reinterpret_cast<double2*>(out + row0);
            dst[0] = make_double2(o[0], o[1]);
            dst[1] = make_double2(o[2], o[3]);
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (r < nr) out[row0 + r] = o[r];
        }
    }
    if (failed) {
        if (lane == 0) atomicExch(err, ERR_WAIT_TIMEOUT);
        for (uint32_t jj = failed_at; jj < n_mine && jj < failed_at + TS_STAGES; ++jj)
            (void)mbar_wait_bounded(&bars[jj % TS_STAGES], (jj / TS_STAGES) & 1u);
    }
}

}  // namespace wgpu
