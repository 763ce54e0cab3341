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
// a block-wide segmented inclusive scan (CUB BlockScan) and emits every segment
// that starts and ends inside the tile.  A segment that crosses tiles leaves a
// tail partial (its owner tile) and head partials (the tiles it continues into);
// the last of those CTAs to finish -- decided by one atomic counter per split
// segment, not a wait -- adds them in tile order and emits.  Every sum is
// therefore formed in one fixed order: results are bitwise reproducible run to
// run, with no floating-point atomics.
//
// The tile/split tables are built once on the host (HostPlan::add) from the
// segment pointer arrays, which never change after set-up.
#pragma once
#include <cstdint>
#include <cub/block/block_scan.cuh>

#include "segplan.hpp"

namespace wgpu {

template <int K>
struct SegItem {
    double v[K];
    int sid;  // id of the segment that starts here (scan: the segment this position belongs to), -1 = none
};

template <int K>
struct SegSumOp {
    __device__ __forceinline__ SegItem<K> operator()(const SegItem<K>& a, const SegItem<K>& b) const {
        if (b.sid >= 0) return b;
        SegItem<K> c;
#pragma unroll
        for (int k = 0; k < K; ++k) c.v[k] = a.v[k] + b.v[k];
        c.sid = a.sid;
        return c;
    }
};

template <int K>
constexpr int sr_items() { return K >= 4 ? 2 : 4; }
template <int K>
constexpr int sr_tile() { return SR_THREADS * sr_items<K>(); }
// resident CTAs per SM the register budget is sized for (no spills at K = 8)
template <int K>
constexpr int sr_min_blocks() { return K >= 8 ? 2 : (K >= 4 ? 3 : (K >= 2 ? 4 : 6)); }
// the scan runs one column at a time over the positions' K-wide values
using SegItem1 = SegItem<1>;

// F provides:
//   using Prob = ...;                 (trivially copyable, <= 256 bytes)
//   const Prob* probs;                (device array)
//   __device__ const uint32_t* seg_ptr(const Prob&) const;
//   __device__ void value(const Prob&, uint32_t pos, double (&v)[K]) const;
//   __device__ void emit(const Prob&, uint32_t seg, const double (&s)[K]) const;
//
// The block scan carries, for every position, the id of the segment it belongs
// to, so the thread holding a segment's last position emits it straight from
// registers; only the 2048-entry head table lives in shared memory.
template <class F, int K>
__global__ void __launch_bounds__(SR_THREADS, sr_min_blocks<K>())
segreduce_kernel(F f, const SRTile* __restrict__ tiles, uint32_t tile_base,
                 const SRSplit* __restrict__ splits, double* __restrict__ head_buf,
                 double* __restrict__ tail_buf, unsigned* __restrict__ counters,
                 const int* __restrict__ skip) {
    constexpr int ITEMS = sr_items<K>();
    constexpr int T = SR_THREADS * ITEMS;
    using Prob = typename F::Prob;
    using Scan = cub::BlockScan<SegItem1, SR_THREADS>;
    __shared__ typename Scan::TempStorage scan_tmp;
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
            double z[K];
#pragma unroll
            for (int k = 0; k < K; ++k) z[k] = 0.0;
            f.emit(prob, s, z);   // empty segment
        }
    }
    __syncthreads();

    // values of this thread's positions, all K columns (index loads shared)
    double val[ITEMS][K];
    int sid[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        uint32_t p = (uint32_t)(tid * ITEMS + i);
        if (p0 + p < p1) {
            f.value(prob, p0 + p, val[i]);
            sid[i] = headseg[p];
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) val[i][k] = 0.0;
            sid[i] = -2;   // past the tile end: never emitted
        }
    }
    // one segmented inclusive scan per column; the carried segment id is the
    // same for every column
#pragma unroll
    for (int k = 0; k < K; ++k) {
        SegItem1 it[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            it[i].v[0] = val[i][k];
            it[i].sid = sid[i];
        }
        if (k > 0) __syncthreads();   // scan_tmp reuse
        Scan(scan_tmp).InclusiveScan(it, it, SegSumOp<1>());
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            val[i][k] = it[i].v[0];
            if (k == K - 1) sid[i] = it[i].sid;
        }
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
        double o[K];
#pragma unroll
        for (int k = 0; k < K; ++k) o[k] = val[i][k];
        if (sg >= 0) {
            if (ptr[sg + 1] <= p1) {
                f.emit(prob, (uint32_t)sg, o);
            } else {   // the owned segment that runs past the tile: tail partial
#pragma unroll
                for (int k = 0; k < K; ++k) tail_buf[(size_t)tile.tail_split * K + k] = o[k];
                __threadfence();
            }
        } else {       // the segment continuing into this tile: head partial
#pragma unroll
            for (int k = 0; k < K; ++k) head_buf[(size_t)gtile * K + k] = o[k];
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
            double tot[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                double v = __ldcg(&tail_buf[(size_t)id * K + k]);
                for (int w = 0; w < SR_THREADS / 32; ++w) v += wsum[w * K + k];
                tot[k] = v;
            }
            Prob pr = (sp.problem == tile.problem) ? prob : f.probs[sp.problem];
            f.emit(pr, sp.seg, tot);
            counters[id] = 0;
        }
        __syncthreads();
    }
}

// Host-side plan of one launch (device arrays).
struct SRPlan {
    int n_tiles = 0;
    int n_splits = 0;
    SRTile* tiles = nullptr;
    SRSplit* splits = nullptr;
    double* head_buf = nullptr;   // n_tiles * K
    double* tail_buf = nullptr;   // n_splits * K
    unsigned* counters = nullptr; // n_splits
    int K = 1;
};

}  // namespace wgpu
