// segsweep.cuh -- deterministic segmented reduction by warp ranges.
//
// The second engine for "sum the entries of each segment" (the first is the
// tile engine of segreduce.cuh, with the same value / emit functors): the
// positions of every problem are cut into fixed ranges of consecutive
// positions, one warp per range, and the warp walks its range in chunks of
// 32 x R positions (lane l holds positions l*R .. l*R+R-1 of the chunk).  A
// host-built bitmap marks the positions where a non-empty segment starts, so
// the warp learns every segment boundary of a chunk from R bits per lane: a
// warp-level segmented scan sums the chunk, every segment that ends in the
// chunk is emitted from registers, and the open segment's partial is carried
// in registers into the next chunk.  There are no block barriers and no
// shared memory: a warp's only dependent waits are its own loads, and the
// next chunk's values are requested before the current chunk is scanned and
// emitted, so a chunk's emit chain (the functor's per-segment loads) overlaps
// the next chunk's streaming loads.
//
// A segment spanning ranges leaves a tail partial (the range it starts in)
// and head partials (the ranges it continues into, a whole range when the
// segment covers it); the last of those warps to finish -- decided by one
// atomic counter per split segment, not a wait -- adds them in range order
// with a fixed shuffle tree and emits.  Every sum has one fixed order, so
// results are bitwise reproducible run to run; no floating-point atomics.
// Empty segments are emitted as zeros by the range holding their position.
//
// The range tables are built once on the host (SSHostPlan::add).
#pragma once
#include "pdl.cuh"
#include <cstdint>

#include "segplan.hpp"

namespace wgpu {

// positions per lane and chunk: 4 for K = 1, 2 for K = 2, 1 for K >= 4
template <int K>
constexpr int ss_items() { return K >= 4 ? 1 : (K >= 2 ? 2 : 4); }
template <int K, class A = double>
constexpr int ss_min_blocks() {
    constexpr int w = K * (int)sizeof(A) / 8;
    return w >= 8 ? 2 : (w >= 4 ? 3 : 4);
}

__device__ __forceinline__ unsigned ss_lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <class F, int K, int R>
__device__ __forceinline__ void ss_load(const F& f, const typename F::Prob& pr, uint32_t c, uint32_t p1, int lane,
                                        typename F::Acc (&v)[R][K]) {
    using A = typename F::Acc;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const uint32_t P = c + (uint32_t)lane * R + i;
        if (P < p1) {
            f.value(pr, P, v[i]);
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) v[i][k] = (A)0;
        }
    }
}

template <class F, int K, int R = ss_items<K>()>
__global__ void __launch_bounds__(SS_THREADS, ss_min_blocks<K, typename F::Acc>())
segsweep_kernel(F f, const SSRange* __restrict__ ranges, uint32_t r_lo, uint32_t r_hi,
                const uint32_t* __restrict__ bits, const uint32_t* __restrict__ nz_ids,
                const uint32_t* __restrict__ empties, const SSSplit* __restrict__ splits,
                double* __restrict__ head_buf, double* __restrict__ tail_buf, unsigned* __restrict__ counters,
                const int* __restrict__ skip) {
    pdl_wait();
    pdl_launch_dependents();
    using Prob = typename F::Prob;
    using A = typename F::Acc;
    constexpr uint32_t CH = 32u * R;
    const unsigned FULL = 0xffffffffu;
    if (skip && *skip) return;
    const int lane = threadIdx.x & 31;
    const uint32_t r = r_lo + blockIdx.x * (SS_THREADS / 32) + (threadIdx.x >> 5);
    if (r >= r_hi) return;   // whole warps
    const SSRange rg = ranges[r];
    const Prob pr = f.probs[rg.problem];
    for (uint32_t e = rg.e_lo + lane; e < rg.e_hi; e += 32) {
        A z[K];
#pragma unroll
        for (int k = 0; k < K; ++k) z[k] = (A)0;
        f.emit(pr, empties[e], z);
    }
    const unsigned lt = ss_lanemask_lt();
    // ordinal of the segment open before the first position: a start at p0
    // (no head split) counts up to o0, a continuing segment is o0 itself
    uint32_t o_base = rg.o0 - (rg.head_split < 0 ? 1u : 0u);
    A carry[K];
#pragma unroll
    for (int k = 0; k < K; ++k) carry[k] = (A)0;
    bool cseen = false;   // a segment start was seen earlier in the range
    A cv[R][K];
    if (rg.p0 < rg.p1) ss_load<F, K, R>(f, pr, rg.p0, rg.p1, lane, cv);
    for (uint32_t c = rg.p0; c < rg.p1; c += CH) {
        const uint32_t cn = c + CH;
        A nv[R][K];
        if (cn < rg.p1) ss_load<F, K, R>(f, pr, cn, rg.p1, lane, nv);   // the next chunk, requested first
        const uint32_t wrel = (c - rg.p0) / 32u;
        const uint32_t word = __ldg(bits + rg.word0 + wrel + ((uint32_t)lane * R) / 32u);
        const uint32_t P0 = c + (uint32_t)lane * R;
        const int nval = P0 >= rg.p1 ? 0 : (int)min((uint32_t)R, rg.p1 - P0);
        uint32_t fl = (word >> (((uint32_t)lane * R) & 31u)) & ((1u << R) - 1u);
        fl &= (1u << nval) - 1u;
        // start flag of the position after this lane's last one
        uint32_t nxt = __shfl_down_sync(FULL, fl, 1) & 1u;
        if (lane == 31) nxt = cn < rg.p1 ? (__ldg(bits + rg.word0 + (cn - rg.p0) / 32u) & 1u) : 0u;
        // (1) the lane's aggregate: the sum after its last start (all items if none)
        A tv[K];
#pragma unroll
        for (int k = 0; k < K; ++k) tv[k] = (A)0;
#pragma unroll
        for (int i = 0; i < R; ++i) {
            if ((fl >> i) & 1u) {
#pragma unroll
                for (int k = 0; k < K; ++k) tv[k] = cv[i][k];
            } else {
#pragma unroll
                for (int k = 0; k < K; ++k) tv[k] += cv[i][k];
            }
        }
        // (2) warp segmented inclusive scan of the lane aggregates
        bool tf = fl != 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            A up[K];
#pragma unroll
            for (int k = 0; k < K; ++k) up[k] = __shfl_up_sync(FULL, tv[k], d);
            const bool uf = __shfl_up_sync(FULL, (int)tf, d) != 0;
            if (lane >= d && !tf) {
#pragma unroll
                for (int k = 0; k < K; ++k) tv[k] += up[k];
                tf = uf;
            }
        }
        A run[K];
#pragma unroll
        for (int k = 0; k < K; ++k) run[k] = __shfl_up_sync(FULL, tv[k], 1);
        bool exf = __shfl_up_sync(FULL, (int)tf, 1) != 0;
        if (lane == 0) {
            exf = false;
#pragma unroll
            for (int k = 0; k < K; ++k) run[k] = (A)0;
        }
        if (!exf) {
#pragma unroll
            for (int k = 0; k < K; ++k) run[k] = carry[k] + run[k];
        }
        bool seen = exf || cseen;
        // starts in the lanes before this one (ordinal bookkeeping)
        uint32_t before = 0, total = 0;
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const unsigned b = __ballot_sync(FULL, (fl >> i) & 1u);
            before += __popc(b & lt);
            total += __popc(b);
        }
        // (3) this lane's items: the running sums, and an emit (or a split
        // partial) at every position that ends a segment piece
        uint32_t cnt = before;
#pragma unroll
        for (int i = 0; i < R; ++i) {
            if (i < nval) {
                if ((fl >> i) & 1u) {
#pragma unroll
                    for (int k = 0; k < K; ++k) run[k] = cv[i][k];
                    seen = true;
                    ++cnt;
                } else {
#pragma unroll
                    for (int k = 0; k < K; ++k) run[k] += cv[i][k];
                }
                const uint32_t P = P0 + i;
                const bool at_end = P + 1 == rg.p1;
                const bool nstart = i + 1 < R ? ((fl >> (i + 1)) & 1u) != 0 : nxt != 0;
                if (at_end || nstart) {
                    if (!seen) {   // the piece of the segment continuing from an earlier range
#pragma unroll
                        for (int k = 0; k < K; ++k) head_buf[(size_t)r * K + k] = (double)run[k];
                        __threadfence();
                    } else if (at_end && rg.tail_split >= 0) {   // the segment runs past the range
#pragma unroll
                        for (int k = 0; k < K; ++k) tail_buf[(size_t)rg.tail_split * K + k] = (double)run[k];
                        __threadfence();
                    } else {
                        const uint32_t o = o_base + cnt;
                        const uint32_t seg = rg.nz_off == SS_IDENTITY ? o : __ldg(nz_ids + rg.nz_off + o);
                        A out[K];
#pragma unroll
                        for (int k = 0; k < K; ++k) out[k] = run[k];
                        f.emit(pr, seg, out);
                    }
                }
            }
        }
        // carry the open segment into the next chunk (a full chunk: lane 31 holds its last position)
#pragma unroll
        for (int k = 0; k < K; ++k) carry[k] = __shfl_sync(FULL, run[k], 31);
        cseen = __shfl_sync(FULL, (int)seen, 31) != 0;
        o_base += total;
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
            for (int k = 0; k < K; ++k) cv[i][k] = nv[i][k];
    }
    __syncwarp();
    // split segments: the last of their ranges to arrive adds the partials in range order
    int fin0 = -1, fin1 = -1;
    if (lane == 0) {
        const int ids[2] = {rg.head_split, rg.tail_split};
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int id = ids[j];
            if (id < 0) continue;
            const SSSplit sp = splits[id];
            const unsigned n_parts = sp.r1 - sp.r0 + 1;
            const unsigned prev = atomicAdd(&counters[id], 1u);
            if (prev == n_parts - 1) (j == 0 ? fin0 : fin1) = id;
        }
    }
    fin0 = __shfl_sync(FULL, fin0, 0);
    fin1 = __shfl_sync(FULL, fin1, 0);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int id = j == 0 ? fin0 : fin1;
        if (id < 0) continue;   // warp-uniform
        __threadfence();
        const SSSplit sp = splits[id];
        double acc[K];
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] = 0.0;
        for (uint32_t t = sp.r0 + 1 + lane; t <= sp.r1; t += 32)
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] += __ldcg(&head_buf[(size_t)t * K + k]);
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(FULL, acc[k], o);
        if (lane == 0) {
            A tot[K];
#pragma unroll
            for (int k = 0; k < K; ++k) tot[k] = (A)(__ldcg(&tail_buf[(size_t)id * K + k]) + acc[k]);
            if (sp.problem == rg.problem) {
                f.emit(pr, sp.seg, tot);
            } else {
                const Prob p2 = f.probs[sp.problem];
                f.emit(p2, sp.seg, tot);
            }
            counters[id] = 0;
        }
    }
}

}  // namespace wgpu
