// xtab.cu -- the weighted cross-tab of a channel pair on the GPU, the first
// step of the additive-Schwarz set-up (the reference accumulates it on the
// host: crates/within/src/domain/cross_tab/accumulate.rs:86-196).
//
// For channels (term a, load la) and (term b, load lb) the cross-tab has one
// cell per observed level pair (a_i, b_i) holding sum_i w_i * la_i * lb_i.
// Sort-and-segment: the observations' keys (a_i << bits_b | b_i) are sorted by
// a stable radix sort carrying the observation index, so every cell's
// observations are contiguous and in observation order; one thread per cell
// then sums them in that order with round-to-nearest multiplies and adds (no
// contraction into fused multiply-adds) -- the same operations, in the same
// order, as the host accumulation, so both give the same bits.  Cells whose
// sum is exactly zero are dropped, as on the host.  The kept cells come back
// as CSR by a and, after a second sort by (b, a), CSC by b; row pointers are
// filled gap by gap, with no atomics.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <thread>
#include <string>
#include <vector>

#include "host.hpp"

namespace wgpu {
namespace {

#define XT_CK(x)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr int XT_THREADS = 256;

// WITHIN_TRACE=1: device and copy times of each cross-tab on stderr
bool xt_trace() {
    static const bool on = [] {
        const char* e = std::getenv("WITHIN_TRACE");
        return e && std::atoi(e) != 0;
    }();
    return on;
}
double xt_now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int bits_for(uint32_t levels) {
    int b = 1;
    while (b < 32 && (1ull << b) < levels) ++b;
    return b;
}

__global__ void k_xt_keys(uint64_t n, const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, int bits_b,
                          uint64_t* __restrict__ key, uint32_t* __restrict__ idx) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        key[i] = ((uint64_t)__ldg(a + i) << bits_b) | __ldg(b + i);
        idx[i] = (uint32_t)i;
    }
}

// 1 where a new cell starts in the sorted keys
__global__ void k_xt_heads(uint64_t n, const uint64_t* __restrict__ key, uint32_t* __restrict__ head) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        head[i] = (i == 0 || key[i] != key[i - 1]) ? 1u : 0u;
}

// start position of every cell (cell_of = inclusive scan of the heads)
__global__ void k_xt_starts(uint64_t n, const uint32_t* __restrict__ head, const uint32_t* __restrict__ cell_of,
                            uint32_t* __restrict__ start) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (head[i]) start[cell_of[i] - 1] = (uint32_t)i;
        if (i == n - 1) start[cell_of[i]] = (uint32_t)n;
    }
}

// one thread per cell: the sum of its observations' w * la * lb in observation
// order (sorted positions start[c] .. start[c + 1]), and whether it is kept
__global__ void k_xt_sums(uint32_t n_cells, const uint32_t* __restrict__ start, const uint32_t* __restrict__ idx,
                          const double* __restrict__ w, const double* __restrict__ la,
                          const double* __restrict__ lb, double* __restrict__ sum, uint32_t* __restrict__ keep) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    const uint32_t p0 = start[c], p1 = start[c + 1];
    double v = 0.0;
    if (!w && !la && !lb) {
        v = (double)(p1 - p0);   // a sum of ones: exact
    } else {
        for (uint32_t p = p0; p < p1; ++p) {
            const uint32_t i = __ldg(idx + p);
            const double wi = w ? __ldg(w + i) : 1.0;
            const double x = la ? __ldg(la + i) : 1.0;
            const double y = lb ? __ldg(lb + i) : 1.0;
            v = __dadd_rn(v, __dmul_rn(__dmul_rn(wi, x), y));
        }
    }
    sum[c] = v;
    keep[c] = v != 0.0 ? 1u : 0u;
}

// compaction of the kept cells: level ids and values (pos = inclusive scan of keep)
__global__ void k_xt_compact(uint32_t n_cells, const uint32_t* __restrict__ start, const uint64_t* __restrict__ key,
                             const double* __restrict__ sum, const uint32_t* __restrict__ keep,
                             const uint32_t* __restrict__ pos, int bits_b, uint32_t* __restrict__ ra,
                             uint32_t* __restrict__ cb, double* __restrict__ val, uint64_t* __restrict__ tkey,
                             uint32_t* __restrict__ tidx, int bits_a) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells || !keep[c]) return;
    const uint32_t k = pos[c] - 1;
    const uint64_t kk = key[start[c]];
    const uint32_t r = (uint32_t)(kk >> bits_b), q = (uint32_t)(kk & ((1ull << bits_b) - 1));
    ra[k] = r;
    cb[k] = q;
    val[k] = sum[c];
    tkey[k] = ((uint64_t)q << bits_a) | r;
    tidx[k] = k;
}

// ptr[r] = first entry whose (sorted) line id is >= r, for r in [0, n_lines]:
// entry k fills the lines after its predecessor's up to its own
__global__ void k_xt_ptr(uint32_t nnz, const uint32_t* __restrict__ line, uint32_t n_lines, uint32_t* __restrict__ ptr) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > nnz) return;
    const uint32_t lo = k == 0 ? 0u : line[k - 1] + 1;
    const uint32_t hi = k == nnz ? n_lines : line[k];
    for (uint32_t r = lo; r <= hi; ++r) ptr[r] = k;
}

__global__ void k_xt_transpose(uint32_t nnz, const uint64_t* __restrict__ tkey, const uint32_t* __restrict__ tidx,
                               const double* __restrict__ val, int bits_a, uint32_t* __restrict__ tcol,
                               uint32_t* __restrict__ trow, double* __restrict__ tval) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    const uint64_t kk = tkey[k];
    tcol[k] = (uint32_t)(kk >> bits_a);
    trow[k] = (uint32_t)(kk & ((1ull << bits_a) - 1));
    tval[k] = val[tidx[k]];
}

// connected components of the cell graph by label propagation with pointer
// jumping: every vertex starts as its own label, every edge hooks the larger
// of its two labels' representatives onto the smaller (atomicMin), then every
// label jumps to its representative's label until both settle; repeated
// until an edge pass sees no two different labels.  Labels only decrease and
// the smallest vertex of a component keeps its own, so the fixed point -- the
// smallest vertex of each component -- is the same whatever the schedule.
__global__ void k_cc_init(uint32_t nv, uint32_t* __restrict__ lab) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < nv) lab[v] = v;
}

__global__ void k_cc_hook(uint32_t nnz, const uint32_t* __restrict__ ra, const uint32_t* __restrict__ cb,
                          uint32_t L_a, uint32_t* lab, int* __restrict__ changed) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    const uint32_t a = lab[ra[k]], b = lab[L_a + cb[k]];
    if (a == b) return;
    atomicMin(&lab[a > b ? a : b], a < b ? a : b);
    *changed = 1;
}

__global__ void k_cc_jump(uint32_t nv, uint32_t* lab) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    uint32_t l = lab[v];
    for (uint32_t t = 0; t < 64; ++t) {   // at most 64 hops a pass; the passes repeat until labels settle
        const uint32_t m = lab[l];
        if (m == l) break;
        l = m;
    }
    lab[v] = l;
}

// all temporaries of one cross-tab carved from a single allocation sized for
// the worst case (cells and kept cells bounded by the observations), so a
// pair pays one allocation and one free
struct DevBuf {
    char* base = nullptr;
    size_t cap = 0, used = 0;
    explicit DevBuf(size_t bytes) : cap(bytes) { XT_CK(cudaMalloc((void**)&base, cap)); }
    template <class T>
    T* get(size_t n) {
        const size_t b = (std::max<size_t>(1, n) * sizeof(T) + 255) / 256 * 256;
        if (used + b > cap) throw std::runtime_error("gpu_cross_tab: scratch plan exceeded");
        T* q = reinterpret_cast<T*>(base + used);
        used += b;
        return q;
    }
    ~DevBuf() { cudaFree(base); }
};

int grid_of(uint64_t n) {
    const uint64_t b = (n + XT_THREADS - 1) / XT_THREADS;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, 148u * 16u));
}

}  // namespace

// Cross-tab of one channel pair; a_dev / b_dev are the two terms' codes
// (internal order), la / lb their loads or nullptr for intercepts, w the
// weights or nullptr.  Synchronous on `st`.
void gpu_cross_tab(uint64_t n, const uint32_t* a_dev, uint32_t L_a, const uint32_t* b_dev, uint32_t L_b,
                   const double* w, const double* la, const double* lb, CrossTab& out, cudaStream_t st) {
    const double t0 = xt_trace() ? xt_now() : 0.0;
    const int bits_a = bits_for(L_a), bits_b = bits_for(L_b);
    if (bits_a + bits_b > 64) throw std::runtime_error("gpu_cross_tab: level ids need more than 64 key bits");
    if (n >= 0xFFFFFFFFull) throw std::runtime_error("gpu_cross_tab: more than 2^32 - 1 observations");
    out.row_ptr.assign((size_t)L_a + 1, 0);
    out.col_ptr.assign((size_t)L_b + 1, 0);
    out.col.clear();
    out.val.clear();
    out.row.clear();
    out.tval.clear();
    out.comp.clear();
    if (n == 0) return;
    // scratch of every step below, with the library's temporary sizes queried for n items
    size_t tb = 0, sb = 0;
    XT_CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint64_t*)nullptr, (uint64_t*)nullptr, (uint32_t*)nullptr,
                                          (uint32_t*)nullptr, (int64_t)n, 0, bits_a + bits_b, st));
    XT_CK(cub::DeviceScan::InclusiveSum(nullptr, sb, (uint32_t*)nullptr, (uint32_t*)nullptr, (int64_t)n, st));
    const size_t pad = 32 * 256;
    DevBuf B(116 * n + 2 * (tb + sb) + 8 * ((size_t)L_a + L_b + 2) + pad);
    uint64_t* key = B.get<uint64_t>(n);
    uint64_t* skey = B.get<uint64_t>(n);
    uint32_t* idx = B.get<uint32_t>(n);
    uint32_t* sidx = B.get<uint32_t>(n);
    k_xt_keys<<<grid_of(n), XT_THREADS, 0, st>>>(n, a_dev, b_dev, bits_b, key, idx);
    XT_CK(cudaGetLastError());
    void* tmp = B.get<char>(tb);
    XT_CK(cub::DeviceRadixSort::SortPairs(tmp, tb, key, skey, idx, sidx, (int64_t)n, 0, bits_a + bits_b, st));
    uint32_t* head = B.get<uint32_t>(n);
    uint32_t* cell_of = B.get<uint32_t>(n);
    k_xt_heads<<<grid_of(n), XT_THREADS, 0, st>>>(n, skey, head);
    XT_CK(cudaGetLastError());
    void* stmp = B.get<char>(sb);
    XT_CK(cub::DeviceScan::InclusiveSum(stmp, sb, head, cell_of, (int64_t)n, st));
    uint32_t n_cells = 0;
    XT_CK(cudaMemcpyAsync(&n_cells, cell_of + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    XT_CK(cudaStreamSynchronize(st));
    uint32_t* start = B.get<uint32_t>((size_t)n_cells + 1);
    k_xt_starts<<<grid_of(n), XT_THREADS, 0, st>>>(n, head, cell_of, start);
    XT_CK(cudaGetLastError());
    double* sum = B.get<double>(n_cells);
    uint32_t* keep = B.get<uint32_t>(n_cells);
    uint32_t* pos = B.get<uint32_t>(n_cells);
    const int cg = (int)((n_cells + XT_THREADS - 1) / XT_THREADS);
    k_xt_sums<<<cg, XT_THREADS, 0, st>>>(n_cells, start, sidx, w, la, lb, sum, keep);
    XT_CK(cudaGetLastError());
    size_t pb = 0;
    XT_CK(cub::DeviceScan::InclusiveSum(nullptr, pb, keep, pos, (int64_t)n_cells, st));
    void* ptmp = B.get<char>(pb);
    XT_CK(cub::DeviceScan::InclusiveSum(ptmp, pb, keep, pos, (int64_t)n_cells, st));
    uint32_t nnz = 0;
    XT_CK(cudaMemcpyAsync(&nnz, pos + (n_cells - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    XT_CK(cudaStreamSynchronize(st));
    uint32_t* ra = B.get<uint32_t>(nnz);
    uint32_t* cb = B.get<uint32_t>(nnz);
    double* val = B.get<double>(nnz);
    uint64_t* tkey = B.get<uint64_t>(nnz);
    uint64_t* stkey = B.get<uint64_t>(nnz);
    uint32_t* tidx = B.get<uint32_t>(nnz);
    uint32_t* stidx = B.get<uint32_t>(nnz);
    k_xt_compact<<<cg, XT_THREADS, 0, st>>>(n_cells, start, skey, sum, keep, pos, bits_b, ra, cb, val, tkey, tidx,
                                            bits_a);
    XT_CK(cudaGetLastError());
    uint32_t* rptr = B.get<uint32_t>((size_t)L_a + 1);
    uint32_t* cptr = B.get<uint32_t>((size_t)L_b + 1);
    const int pg = (int)(((uint64_t)nnz + 1 + XT_THREADS - 1) / XT_THREADS);
    k_xt_ptr<<<pg, XT_THREADS, 0, st>>>(nnz, ra, L_a, rptr);
    XT_CK(cudaGetLastError());
    uint32_t* tcol = B.get<uint32_t>(nnz);
    uint32_t* trow = B.get<uint32_t>(nnz);
    double* tval = B.get<double>(nnz);
    if (nnz) {
        size_t t2 = 0;
        XT_CK(cub::DeviceRadixSort::SortPairs(nullptr, t2, tkey, stkey, tidx, stidx, (int64_t)nnz, 0, bits_a + bits_b,
                                              st));
        void* tmp2 = B.get<char>(t2);
        XT_CK(cub::DeviceRadixSort::SortPairs(tmp2, t2, tkey, stkey, tidx, stidx, (int64_t)nnz, 0, bits_a + bits_b,
                                              st));
        k_xt_transpose<<<(nnz + XT_THREADS - 1) / XT_THREADS, XT_THREADS, 0, st>>>(nnz, stkey, stidx, val, bits_a,
                                                                                   tcol, trow, tval);
        XT_CK(cudaGetLastError());
    }
    k_xt_ptr<<<pg, XT_THREADS, 0, st>>>(nnz, tcol, L_b, cptr);
    XT_CK(cudaGetLastError());
    // connected components over the kept cells
    const uint32_t nv = L_a + L_b;
    uint32_t* lab = B.get<uint32_t>(nv);
    int* changed = B.get<int>(1);
    k_cc_init<<<(nv + XT_THREADS - 1) / XT_THREADS, XT_THREADS, 0, st>>>(nv, lab);
    XT_CK(cudaGetLastError());
    for (uint32_t it = 0;; ++it) {
        if (it > nv) throw std::runtime_error("gpu_cross_tab: components did not settle");
        int h_changed = 0;
        XT_CK(cudaMemsetAsync(changed, 0, sizeof(int), st));
        if (nnz)
            k_cc_hook<<<(nnz + XT_THREADS - 1) / XT_THREADS, XT_THREADS, 0, st>>>(nnz, ra, cb, L_a, lab, changed);
        XT_CK(cudaGetLastError());
        k_cc_jump<<<(nv + XT_THREADS - 1) / XT_THREADS, XT_THREADS, 0, st>>>(nv, lab);
        XT_CK(cudaGetLastError());
        XT_CK(cudaMemcpyAsync(&h_changed, changed, sizeof(int), cudaMemcpyDeviceToHost, st));
        XT_CK(cudaStreamSynchronize(st));
        if (!h_changed) break;
    }
    out.comp.resize(nv);
    if (xt_trace()) XT_CK(cudaStreamSynchronize(st));   // so the trace splits device and copy time
    const double t_dev = xt_trace() ? xt_now() : 0.0;
    {   // fresh host arrays side by side (their first-touch page faults dominate one thread's resize)
        std::thread a([&] { out.col.resize(nnz); }), b([&] { out.val.resize(nnz); }),
            c([&] { out.row.resize(nnz); });
        out.tval.resize(nnz);
        a.join();
        b.join();
        c.join();
    }
    XT_CK(cudaMemcpyAsync(out.row_ptr.data(), rptr, ((size_t)L_a + 1) * 4, cudaMemcpyDeviceToHost, st));
    XT_CK(cudaMemcpyAsync(out.col_ptr.data(), cptr, ((size_t)L_b + 1) * 4, cudaMemcpyDeviceToHost, st));
    XT_CK(cudaMemcpyAsync(out.comp.data(), lab, (size_t)nv * 4, cudaMemcpyDeviceToHost, st));
    if (nnz) {
        XT_CK(cudaMemcpyAsync(out.col.data(), cb, (size_t)nnz * 4, cudaMemcpyDeviceToHost, st));
        XT_CK(cudaMemcpyAsync(out.val.data(), val, (size_t)nnz * 8, cudaMemcpyDeviceToHost, st));
        XT_CK(cudaMemcpyAsync(out.row.data(), trow, (size_t)nnz * 4, cudaMemcpyDeviceToHost, st));
        XT_CK(cudaMemcpyAsync(out.tval.data(), tval, (size_t)nnz * 8, cudaMemcpyDeviceToHost, st));
    }
    XT_CK(cudaStreamSynchronize(st));
    if (xt_trace())
        fprintf(stderr, "[within trace]   GPU cross-tab %u x %u, %u cells: device %.3f ms, host copies %.3f ms\n", L_a,
                L_b, nnz, (t_dev - t0) * 1e3, (xt_now() - t_dev) * 1e3);
}

}  // namespace wgpu
