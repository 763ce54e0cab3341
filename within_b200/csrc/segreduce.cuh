// segreduce.cuh -- deterministic, load-balanced segmented reduction.
//
// One engine serves every "sum the entries of each segment" step of the solve:
// the adjoint scatter D^T u (segments = levels of a term, positions = the
// term's level-sorted observation order), the cross-block SpMVs of the block
// elimination (segments = CSR rows, positions = non-zeros), the Schwarz
// restrict/mean/prolongation combines and the rounds of the triangular solves.
//
// Positions are cut into fixed tiles of T = 256*ITEMS entries, one CTA per
// tile, so work is balanced no matter how the segment lengths are distributed
// (a Pareto firm of 10^6 rows costs the same per row as a worker of 10).  A CTA
// loads its tile (coalesced where the value functor reads contiguously), runs
// a block-wide segmented inclusive scan over all K columns at once (thread
// sums, a warp shuffle scan, one shared-memory exchange of the warp
// aggregates) and emits every segment that starts and ends inside the tile.  A segment that crosses tiles leaves a
// tail partial (its owner tile) and head partials (the tiles it continues into);
// the last of those CTAs to finish -- decided by one atomic counter per split
// segment, not a wait -- adds them in tile order and emits.  Every sum is
// therefore formed in one fixed order: results are bitwise reproducible run to
// run, with no floating-point atomics.
//
// The tile/split tables are built once on the host (HostPlan::add) from the
// segment pointer arrays, which never change after set-up.
#pragma once
#include "pdl.cuh"
#include <cstdint>

#include "segplan.hpp"

namespace wgpu {

template <int K>
constexpr int sr_items() { return K >= 8 ? 2 : 4; }
template <int K>
constexpr int sr_tile() { return SR_THREADS * sr_items<K>(); }
// Wide tiles (4x the items per thread, K <= 2) for problems of long segments
// (restrict / means / kept sums of a few huge subdomains, C^T rows of kept
// levels with many eliminated neighbours, the level-sorted rest terms): a
// tile of mostly interior positions pays the fixed per-tile cost (barriers,
// segment-start table, split bookkeeping) once per 4x more positions, and
// each thread keeps 4x more independent loads in flight.
template <int K>
constexpr int sr_items_wide() { return K == 1 ? 16 : (K == 2 ? 8 : sr_items<K>()); }
template <int K>
constexpr int sr_tile_wide() { return SR_THREADS * sr_items_wide<K>(); }
// the mean segment length from which a plan may take wide tiles (a tuning
// choice, within_tuning.wide_mean_len; off unless chosen)
constexpr uint32_t SR_WIDE_MEAN_LEN = 64;
// resident CTAs per SM the register budget is sized for (no spills at K = 8)
// (the register footprint scales with K x the accumulator width)
template <int K, class A = double>
constexpr int sr_min_blocks() {
    constexpr int w = K * (int)sizeof(A) / 8;
    return w >= 8 ? 2 : (w >= 4 ? 3 : (w >= 2 ? 4 : 6));
}

// F provides:
//   using Prob = ...;                 (trivially copyable, <= 256 bytes)
//   const Prob* probs;                (device array)
//   __device__ const uint32_t* seg_ptr(const Prob&) const;
//   using Acc = double | float;       (register type of the values and the scan)
//   __device__ void value(const Prob&, uint32_t pos, Acc (&v)[K]) const;
//   __device__ void emit(const Prob&, uint32_t seg, const Acc (&s)[K]) const;
// Split-segment partials cross tiles in double whatever Acc is.
//
// The scan carries, for every position, the id of the segment it belongs to
// (-1: the segment continuing from the previous tile), so the thread holding
// a segment's last position emits it straight from registers; the scan's
// combine is "a segment start resets the sum", and the id >= 0 of the last
// start doubles as the reset flag.
template <class F, int K, int ITEMS = sr_items<K>()>
__global__ void __launch_bounds__(SR_THREADS, (ITEMS > sr_items<K>() ? 2 : sr_min_blocks<K, typename F::Acc>()))
segreduce_kernel(F f, const SRTile* __restrict__ tiles, uint32_t tile_base,
                 const SRSplit* __restrict__ splits, double* __restrict__ head_buf,
                 double* __restrict__ tail_buf, unsigned* __restrict__ counters,
                 const int* __restrict__ skip) {
    pdl_wait();
    pdl_launch_dependents();
    constexpr int T = SR_THREADS * ITEMS;
    using Prob = typename F::Prob;
    using A = typename F::Acc;
    constexpr int NW = SR_THREADS / 32;
    __shared__ A wagg[NW][K];
    __shared__ int wsid[NW];
    __shared__ int headseg[T + 1];
    __shared__ double wsum[(SR_THREADS / 32) * K];
    __shared__ SRTile tile;
    __shared__ Prob prob;
    __shared__ int last_split[2];

    if (skip && *skip) return;
    const int tid = threadIdx.x;
    const uint32_t gtile = tile_base + blockIdx.x;   // global tile id
    if (tid == 0) {
        tile = tiles[gtile];
        prob = f.probs[tile.problem];
    }
    for (int i = tid; i <= T; i += SR_THREADS) headseg[i] = -1;
    __syncthreads();
    const uint32_t p0 = tile.p0, p1 = tile.p1;
    const uint32_t* ptr = f.seg_ptr(prob);
    for (uint32_t s = tile.own_lo + tid; s < tile.own_hi; s += SR_THREADS) {
        uint32_t a = ptr[s], b = ptr[s + 1];
        if (b > a) {
            headseg[a - p0] = (int)s;
        } else {
            A z[K];
#pragma unroll
            for (int k = 0; k < K; ++k) z[k] = (A)0;
            f.emit(prob, s, z);   // empty segment
        }
    }
    __syncthreads();

    // values of this thread's positions, all K columns (index loads shared)
    A val[ITEMS][K];
    int sid[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        uint32_t p = (uint32_t)(tid * ITEMS + i);
        if (p0 + p < p1) {
            f.value(prob, p0 + p, val[i]);
            sid[i] = headseg[p];
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) val[i][k] = (A)0;
            sid[i] = -2;   // past the tile end: never emitted
        }
    }
    // segmented inclusive scan of all K columns: (1) the thread's own items,
    const unsigned FULL = 0xffffffffu;
    const int lane = tid & 31, wid = tid >> 5;
    int ts = -1;   // id of the thread's last segment start, -1 = none
    A tv[K];
#pragma unroll
    for (int k = 0; k < K; ++k) tv[k] = (A)0;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        if (sid[i] >= 0) {
            ts = sid[i];
#pragma unroll
            for (int k = 0; k < K; ++k) tv[k] = val[i][k];
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) tv[k] += val[i][k];
        }
    }
    // (2) the warp (shuffle tree),
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        A up[K];
#pragma unroll
        for (int k = 0; k < K; ++k) up[k] = __shfl_up_sync(FULL, tv[k], d);
        const int us = __shfl_up_sync(FULL, ts, d);
        if (lane >= d && ts < 0) {
            ts = us;
#pragma unroll
            for (int k = 0; k < K; ++k) tv[k] += up[k];
        }
    }
    A ex[K];
#pragma unroll
    for (int k = 0; k < K; ++k) ex[k] = __shfl_up_sync(FULL, tv[k], 1);
    int exs = __shfl_up_sync(FULL, ts, 1);
    if (lane == 0) {
        exs = -1;
#pragma unroll
        for (int k = 0; k < K; ++k) ex[k] = (A)0;
    }
    if (lane == 31) {
        wsid[wid] = ts;
#pragma unroll
        for (int k = 0; k < K; ++k) wagg[wid][k] = tv[k];
    }
    __syncthreads();
    // (3) the warps before this one, in warp order
    int cs = -1;
    A cv[K];
#pragma unroll
    for (int k = 0; k < K; ++k) cv[k] = (A)0;
    for (int q = 0; q < wid; ++q) {
        if (wsid[q] >= 0) {
            cs = wsid[q];
#pragma unroll
            for (int k = 0; k < K; ++k) cv[k] = wagg[q][k];
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) cv[k] += wagg[q][k];
        }
    }
    // carry into this thread, then its items again
    int rs = exs >= 0 ? exs : cs;
    A run[K];
#pragma unroll
    for (int k = 0; k < K; ++k) run[k] = exs >= 0 ? ex[k] : cv[k] + ex[k];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        if (sid[i] >= 0) {
            rs = sid[i];
#pragma unroll
            for (int k = 0; k < K; ++k) run[k] = val[i][k];
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) run[k] += val[i][k];
        }
#pragma unroll
        for (int k = 0; k < K; ++k) val[i][k] = run[k];
        if (sid[i] != -2) sid[i] = rs;
    }

    // emit at the last position of each segment piece held by this thread
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint32_t p = (uint32_t)(tid * ITEMS + i);
        const uint32_t P = p0 + p;
        if (P >= p1) continue;
        const bool last = (P + 1 == p1) || headseg[p + 1] >= 0;
        if (!last) continue;
        const int sg = sid[i];
        A o[K];
#pragma unroll
        for (int k = 0; k < K; ++k) o[k] = val[i][k];
        if (sg >= 0) {
            if (ptr[sg + 1] <= p1) {
                f.emit(prob, (uint32_t)sg, o);
            } else {   // the owned segment that runs past the tile: tail partial
#pragma unroll
                for (int k = 0; k < K; ++k) tail_buf[(size_t)tile.tail_split * K + k] = (double)o[k];
                __threadfence();
            }
        } else {       // the segment continuing into this tile: head partial
#pragma unroll
            for (int k = 0; k < K; ++k) head_buf[(size_t)gtile * K + k] = (double)o[k];
            __threadfence();
        }
    }
    __syncthreads();
    if (tid == 0) {
        int ids[2] = {tile.cont_split, tile.tail_split};
        for (int j = 0; j < 2; ++j) {
            last_split[j] = -1;
            int id = ids[j];
            if (id < 0) continue;
            const SRSplit sp = splits[id];
            unsigned total = sp.t1 - sp.t0 + 1;
            unsigned prev = atomicAdd(&counters[id], 1u);
            if (prev == total - 1) last_split[j] = id;
        }
    }
    __syncthreads();
    // The finishing CTA adds the tail partial and the head partials of the
    // split in tile order: thread i takes tiles t0+1+i, t0+1+i+256, ..., then a
    // fixed shuffle tree -- the same order on every run.
    for (int j = 0; j < 2; ++j) {
        const int id = last_split[j];
        if (id < 0) continue;   // uniform across the block (shared)
        __threadfence();
        const SRSplit sp = splits[id];
        double acc[K];
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] = 0.0;
        for (uint32_t t = sp.t0 + 1 + tid; t <= sp.t1; t += SR_THREADS)
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] += __ldcg(&head_buf[(size_t)t * K + k]);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double v = acc[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if ((tid & 31) == 0) wsum[(tid >> 5) * K + k] = v;
        }
        __syncthreads();
        if (tid == 0) {
            A tot[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                double v = __ldcg(&tail_buf[(size_t)id * K + k]);
                for (int w = 0; w < SR_THREADS / 32; ++w) v += wsum[w * K + k];
                tot[k] = (A)v;
            }
            Prob pr = (sp.problem == tile.problem) ? prob : f.probs[sp.problem];
            f.emit(pr, sp.seg, tot);
            counters[id] = 0;
        }
        __syncthreads();
    }
}

// Sum of positions [a, b) of one segment by one thread, in position order.
// Four positions' values are requested before any is added, so four load
// chains (index, value, gathered operand) are in flight at once; the adds
// still run in position order, so the sum has the bits of a plain loop.
template <class F, int K>
__device__ __forceinline__ void seg_sum(const F& f, const typename F::Prob& pr, uint32_t a, uint32_t b,
                                        typename F::Acc (&acc)[K]) {
    using A = typename F::Acc;
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = (A)0;
    uint32_t q = a;
    for (; q + 4 <= b; q += 4) {
        A v0[K], v1[K], v2[K], v3[K];
        f.value(pr, q, v0);
        f.value(pr, q + 1, v1);
        f.value(pr, q + 2, v2);
        f.value(pr, q + 3, v3);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            acc[k] += v0[k];
            acc[k] += v1[k];
            acc[k] += v2[k];
            acc[k] += v3[k];
        }
    }
    for (; q < b; ++q) {
        A v[K];
        f.value(pr, q, v);
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += v[k];
    }
}

// One thread per segment, for a problem whose segments are all short (at
// most SEGT_MAX_LEN positions, as the rows of C, the DOFs' slot lists and the
// factor rows of most elimination rounds are): each thread sums its
// segment's positions in order and emits, with no tile barrier, scan or split
// bookkeeping.  The order is fixed, so results are bitwise reproducible.
constexpr uint32_t SEGT_MAX_LEN = 32;
constexpr int SEGT_THREADS = 256;

template <class F, int K>
__global__ void __launch_bounds__(SEGT_THREADS)
segthread_kernel(F f, uint32_t prob, uint32_t n_seg, const int* __restrict__ skip) {
    pdl_wait();
    pdl_launch_dependents();
    using A = typename F::Acc;
    if (skip && *skip) return;
    const uint32_t sg = blockIdx.x * SEGT_THREADS + threadIdx.x;
    if (sg >= n_seg) return;
    const typename F::Prob pr = f.probs[prob];
    const uint32_t* ptr = f.seg_ptr(pr);
    const uint32_t a = __ldg(ptr + sg), b = __ldg(ptr + sg + 1);
    A acc[K];
    seg_sum<F, K>(f, pr, a, b, acc);
    f.emit(pr, sg, acc);
}

// G lanes per segment, for a problem whose segments are all short (at most
// SEGT_MAX_LEN positions, as the rows of C are): the G lanes of a group read
// consecutive positions of their segment (coalesced across the warp), lane j
// summing positions j, j + G, ... in order (up to four values requested
// before any is added), then a fixed xor tree adds the G lane sums and the
// group's first lane emits.  Every sum has one fixed order, so results are
// bitwise reproducible (they differ in the last bits from segthread_kernel's
// sequential sums).
template <class F, int K, int G>
__global__ void __launch_bounds__(SEGT_THREADS)
segvec_kernel(F f, uint32_t prob, uint32_t n_seg, const int* __restrict__ skip) {
    pdl_wait();
    pdl_launch_dependents();
    static_assert(G >= 2 && G <= 32 && (G & (G - 1)) == 0, "lanes per segment: a power of two up to 32");
    using A = typename F::Acc;
    if (skip && *skip) return;
    const unsigned FULL = 0xffffffffu;
    const uint32_t t = blockIdx.x * SEGT_THREADS + threadIdx.x;
    const uint32_t sg = t / G, j = t % G;
    const bool valid = sg < n_seg;   // every lane of the warp reaches the shuffles
    const typename F::Prob pr = f.probs[prob];
    A acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = (A)0;
    if (valid) {
        const uint32_t* ptr = f.seg_ptr(pr);
        const uint32_t a = __ldg(ptr + sg), b = __ldg(ptr + sg + 1);
        uint32_t q = a + j;
        for (; q + 3 * G < b; q += 4 * G) {
            A v0[K], v1[K], v2[K], v3[K];
            f.value(pr, q, v0);
            f.value(pr, q + G, v1);
            f.value(pr, q + 2 * G, v2);
            f.value(pr, q + 3 * G, v3);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                acc[k] += v0[k];
                acc[k] += v1[k];
                acc[k] += v2[k];
                acc[k] += v3[k];
            }
        }
        for (; q < b; q += G) {
            A v[K];
            f.value(pr, q, v);
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] += v[k];
        }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += __shfl_xor_sync(FULL, acc[k], o);
    if (valid && j == 0) f.emit(pr, sg, acc);
}

// lanes per segment for a plan of mean segment length `mean` (segvec_kernel):
// about two positions per lane, 0 = one thread per segment
inline int segvec_lanes(double mean) {
    int g = 1;
    while (g < 32 && 2.0 * g < mean) g *= 2;
    return g >= 4 ? g : 0;
}

// A run of consecutive elimination rounds whose segments are all short and
// few (the small tail of a round-scheduled factor: rounds of a few hundred
// rows each): one block walks the rounds in order (forward) or in reverse
// (backward), one thread per segment as in segthread_kernel, with a block
// barrier between rounds -- one launch instead of one per round.  The rounds
// are problems r_lo..r_hi-1 of f.probs; round_rows[r] is round r's segment
// count.  Each segment is summed in the order segthread_kernel uses, so the
// results are bitwise the same.
constexpr int RF_THREADS = 1024;
constexpr uint32_t RF_MAX_ROWS = 4 * RF_THREADS;   // rows of a round the fused launch takes

template <class F, int K>
__global__ void __launch_bounds__(RF_THREADS)
rounds_fused_kernel(F f, const uint32_t* __restrict__ round_rows, uint32_t r_lo, uint32_t r_hi, int backward,
                    const int* __restrict__ skip) {
    pdl_wait();
    pdl_launch_dependents();
    using A = typename F::Acc;
    if (skip && *skip) return;
    for (uint32_t i = 0; i < r_hi - r_lo; ++i) {
        const uint32_t r = backward ? r_hi - 1 - i : r_lo + i;
        const typename F::Prob pr = f.probs[r];
        const uint32_t* ptr = f.seg_ptr(pr);
        const uint32_t n_seg = round_rows[r];
        for (uint32_t sg = threadIdx.x; sg < n_seg; sg += RF_THREADS) {
            const uint32_t a = __ldg(ptr + sg), b = __ldg(ptr + sg + 1);
            A acc[K];
            seg_sum<F, K>(f, pr, a, b, acc);
            f.emit(pr, sg, acc);
        }
        __syncthreads();   // the next round reads this round's results
    }
}

// the longest segment of a pointer array (host)
inline uint32_t seg_max_len(const uint32_t* ptr, size_t n_seg) {
    uint32_t m = 0;
    for (size_t i = 0; i < n_seg; ++i) m = ptr[i + 1] - ptr[i] > m ? ptr[i + 1] - ptr[i] : m;
    return m;
}

}  // namespace wgpu
