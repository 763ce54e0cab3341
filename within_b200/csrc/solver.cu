// solver.cu -- the Solver (crates/within/src/solver.rs) on one B200: set-up,
// the device-resident LSMR loop and the C ABI declared in include/within_gpu.h.
//
// A solve of k right-hand sides runs as one multi-RHS modified LSMR
// (crates/schwarz-precond/src/lsmr.rs:206-295): every iteration is a fixed
// sequence of kernels on one stream --
//   gather+update (u <- A v + s u, beta)      k_gather_update
//   scatter A^T u with the p~ epilogue       segreduce<ScatterF>, one launch
//   preconditioner v = M^-1 p~               diagonal kernel / Schwarz chain
//   alpha, Givens recurrences, stop test     k_alpha_step (last block)
//   v, h, h_bar, x update                    k_solution_update
// -- with all scalar state on the device, so the host never waits inside an
// iteration.  Two iterations (both state parities) form the body of a CUDA
// graph with a conditional WHILE node, so a solve is one graph launch and one
// host wait; a finished column stops updating and once every column has
// finished the kernels return at entry.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <functional>
#include <future>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/within_gpu.h"
#include "host.hpp"
#include "host_pool.hpp"
#include "kernels.cuh"
#include "refine.cuh"
#include "rowsweep.cuh"
#include "tsweep.cuh"

using namespace wgpu;

namespace wgpu {
void gpu_cross_tab(uint64_t n, const uint32_t* a_dev, uint32_t L_a, const uint32_t* b_dev, uint32_t L_b,
                   const double* w, const double* la, const double* lb, CrossTab& out, cudaStream_t st);
}

namespace {

thread_local std::string g_err;
thread_local uint64_t g_launches = 0;

#define CK(x)                                                                          \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess)                                                         \
            throw WError(ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));   \
    } while (0)

// WITHIN_TRACE=1: host-side phase times of the set-up and of the lazy first
// use of each column bucket, one line each on stderr (a diagnostic; no effect
// on results)
bool trace_on() {
    static const bool on = [] {
        const char* e = getenv("WITHIN_TRACE");
        return e && atoi(e) != 0;
    }();
    return on;
}
double now_s();
struct PhaseTrace {
    const char* what;
    double t0;
    explicit PhaseTrace(const char* w) : what(w), t0(trace_on() ? now_s() : 0.0) {}
    void done() {
        if (trace_on() && what) fprintf(stderr, "[within trace] %s %.3f ms\n", what, (now_s() - t0) * 1e3);
        what = nullptr;
    }
    ~PhaseTrace() { done(); }
};

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int grid_for(uint64_t n, int threads, int cap) {
    uint64_t b = (n + threads - 1) / threads;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)cap));
}

// Simple owner of device allocations.
struct Arena {
    std::vector<void*> ptrs;
    template <class T>
    T* alloc(size_t n) {
        if (n == 0) n = 1;
        void* p = nullptr;
        CK(cudaMalloc(&p, n * sizeof(T)));
        CK(cudaMemset(p, 0, n * sizeof(T)));
        ptrs.push_back(p);
        return (T*)p;
    }
    template <class T>
    T* upload(const std::vector<T>& v) {
        if (v.empty()) return alloc<T>(1);
        void* p = nullptr;
        CK(cudaMalloc(&p, v.size() * sizeof(T)));
        ptrs.push_back(p);
        CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
        return (T*)p;
    }
    ~Arena() {
        for (void* p : ptrs) cudaFree(p);
    }
};

// Many host arrays uploaded into one device allocation of the arena (each
// at a 256-byte aligned offset; empty arrays get a zeroed slot): one
// cudaMalloc instead of one per array.
struct UploadBatch {
    struct Item {
        const void* src;
        size_t bytes, off;
        std::function<void(char*)> set;
    };
    std::vector<Item> items;
    size_t total = 0;
    template <class T, class P>
    void add(P*& dst, const std::vector<T>& v) {
        const size_t b = v.size() * sizeof(T);
        items.push_back({v.data(), b, total, [&dst](char* p) { dst = reinterpret_cast<P*>(p); }});
        total += (std::max<size_t>(b, 1) + 255) / 256 * 256;
    }
    void commit(Arena& A) {
        char* base = nullptr;
        CK(cudaMalloc(&base, std::max<size_t>(total, 256)));
        A.ptrs.push_back(base);
        CK(cudaMemset(base, 0, std::max<size_t>(total, 256)));
        for (Item& it : items) {
            it.set(base + it.off);
            if (it.bytes) CK(cudaMemcpy(base + it.off, it.src, it.bytes, cudaMemcpyHostToDevice));
        }
    }
};

// A segmented-reduction launch set on device.
struct DevPlan {
    SRTile* tiles = nullptr;
    SRSplit* splits = nullptr;
    double* head = nullptr;
    double* tail = nullptr;
    unsigned* counters = nullptr;
    uint32_t n_tiles = 0;
    uint32_t n_splits = 0;
    bool wide = false;   // tiles of sr_tile_wide<K>() positions (else sr_tile<K>())
    std::vector<uint32_t> range_lo, range_hi;   // tile ranges (per round, for round plans)
    // warp-range plan (segsweep.cuh): n_tiles counts ranges, head holds one
    // partial per range, tail / counters one per split segment
    bool ss = false;
    SSRange* ranges = nullptr;
    SSSplit* ss_splits = nullptr;
    uint32_t* bits = nullptr;
    uint32_t* nz_ids = nullptr;
    uint32_t* empties = nullptr;
};

// The per-solver choices of kernel variants and factor stop rules
// (within_tuning of the C ABI), resolved once when the solver is built:
// explicit fields of the caller's record, else the WITHIN_* environment
// overrides, else the defaults.  Every choice is a function of the design and
// this record only, so summation orders -- and results -- are reproducible.
struct Tuning {
    bool staged = true;          // staged (TMA) row sweep and gather where they apply
    // plans whose segments average this many positions take wide tiles; off by
    // default (on the 10M-row panel wide tiles made C^T, restrict, means and
    // kept sums 1.5-2x slower: two blocks per SM hide less latency)
    uint32_t wide_mean_len = UINT32_MAX;
    bool fuse_rounds = true;     // the small tail of elimination rounds in one block
    bool segthread = true;       // one thread per segment where every segment is short
    // segmented reductions by warp ranges (segsweep.cuh) instead of block
    // tiles: 1 = C^T and the adjoint's combines of single-column solves (rows
    // of ~10-1000 positions, measured faster on the 10M-row panel; at four
    // columns a lane holds one position and C^T was slower), 2 = every tile
    // plan at every column count (restrict, means, kept sums, rounds, ...
    // measured slower), 0 = none
    int warp_ranges = 1;
    // cross-tabs of the additive-Schwarz set-up on the GPU (xtab.cu): 1 for
    // designs of at least XTAB_MIN_OBS observations, 2 always, 0 never
    int gpu_cross_tab = 1;
    // C's rows (all short) by groups of lanes (segvec_kernel) instead of one thread each
    bool vector_rows = false;
};
constexpr uint64_t XTAB_MIN_OBS = 1ull << 18;

Tuning resolve_tuning(const within_tuning* t) {
    Tuning r;
    if (t) {
        r.staged = t->staged_sweep != 0;
        r.wide_mean_len = t->wide_mean_len;
        r.fuse_rounds = t->fuse_rounds != 0;
        r.segthread = t->thread_per_segment != 0;
        r.warp_ranges = t->warp_ranges;
        r.gpu_cross_tab = t->gpu_cross_tab;
        r.vector_rows = t->vector_rows != 0;
        return r;
    }
    if (const char* e = getenv("WITHIN_TSWEEP")) r.staged = atoi(e) != 0;
    if (const char* e = getenv("WITHIN_WIDE_TILES"))
        if (atoi(e) == 0) r.wide_mean_len = UINT32_MAX;
    if (const char* e = getenv("WITHIN_FUSE_ROUNDS")) r.fuse_rounds = atoi(e) != 0;
    if (const char* e = getenv("WITHIN_SEGTHREAD")) r.segthread = atoi(e) != 0;
    if (const char* e = getenv("WITHIN_WARP_RANGES")) r.warp_ranges = atoi(e);
    if (const char* e = getenv("WITHIN_GPU_XTAB")) r.gpu_cross_tab = atoi(e);
    if (const char* e = getenv("WITHIN_VECTOR_ROWS")) r.vector_rows = atoi(e) != 0;
    return r;
}

// Tile size of a plan: wide tiles when K <= 2 and its segments average
// wide_mean_len positions or more.  Fixed by the design and the tuning, so
// the summation order is too.
bool plan_wide(int K, uint64_t positions, uint64_t segments, uint32_t wide_mean_len) {
    if (K > 2 || wide_mean_len == UINT32_MAX) return false;
    return segments > 0 && positions >= (uint64_t)wide_mean_len * segments;
}
int plan_tile(int K, bool wide) {
    if (wide) return K == 1 ? sr_tile_wide<1>() : sr_tile_wide<2>();
    return K == 1 ? sr_tile<1>() : K == 2 ? sr_tile<2>() : K == 4 ? sr_tile<4>() : sr_tile<8>();
}

DevPlan make_plan(Arena& A, const HostPlan& hp, int K) {
    DevPlan d;
    d.n_tiles = (uint32_t)hp.tiles.size();
    d.n_splits = (uint32_t)hp.splits.size();
    d.tiles = A.upload(hp.tiles);
    d.splits = A.upload(hp.splits);
    d.head = A.alloc<double>((size_t)d.n_tiles * K);
    d.tail = A.alloc<double>(std::max<size_t>(1, hp.splits.size()) * K);
    d.counters = A.alloc<unsigned>(std::max<size_t>(1, hp.splits.size()));
    return d;
}

DevPlan make_ss_plan(Arena& A, const SSHostPlan& hp, int K) {
    DevPlan d;
    d.ss = true;
    d.n_tiles = (uint32_t)hp.ranges.size();
    d.n_splits = (uint32_t)hp.splits.size();
    d.ranges = A.upload(hp.ranges);
    d.ss_splits = A.upload(hp.splits);
    d.bits = A.upload(hp.bits);
    d.nz_ids = hp.nz_ids.empty() ? nullptr : A.upload(hp.nz_ids);
    d.empties = hp.empties.empty() ? nullptr : A.upload(hp.empties);
    d.head = A.alloc<double>(std::max<size_t>(1, hp.ranges.size()) * K);
    d.tail = A.alloc<double>(std::max<size_t>(1, hp.splits.size()) * K);
    d.counters = A.alloc<unsigned>(std::max<size_t>(1, hp.splits.size()));
    return d;
}

// Warps a warp-range plan is cut for: one wave of the kernel's resident warps.
uint32_t ss_target_warps(int K) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    const int blocks = K >= 8 ? 2 : (K >= 4 ? 3 : 4);
    return (uint32_t)(sms * blocks * (SS_THREADS / 32));
}

// Kernels launched with programmatic stream serialisation (pdl.cuh): each
// may be scheduled while its predecessor's last blocks run and waits for it
// in-kernel.  Process-wide; WITHIN_PDL=0 launches in plain stream order.
bool pdl_on() {
    static const bool on = [] {
        const char* e = getenv("WITHIN_PDL");
        return e ? atoi(e) != 0 : true;
    }();
    return on;
}

// c_pdl_early on the current device (once per device; WITHIN_PDL_EARLY=1)
void pdl_setup(int dev) {
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> g(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return;
    const char* e = getenv("WITHIN_PDL_EARLY");
    const int v = e ? atoi(e) : 0;
    CK(cudaMemcpyToSymbol(c_pdl_early, &v, sizeof(int)));
    done.push_back(dev);
}

template <class... KArgs, class... Args>
void launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_on() ? 1 : 0;
    CK(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
}

template <class F, int K>
void launch_segthread(const F& f, uint32_t prob, uint32_t n_seg, const int* skip, cudaStream_t st) {
    if (!n_seg) return;
    launch_k(segthread_kernel<F, K>, (n_seg + SEGT_THREADS - 1) / SEGT_THREADS, SEGT_THREADS, 0, st, f, prob, n_seg,
                                                                                                skip);
    ++g_launches;
}

template <class F, int K>
void launch_segvec(const F& f, uint32_t prob, uint32_t n_seg, int lanes, const int* skip, cudaStream_t st) {
    if (!n_seg) return;
    const uint64_t threads = (uint64_t)n_seg * lanes;
    const unsigned grid = (unsigned)((threads + SEGT_THREADS - 1) / SEGT_THREADS);
    switch (lanes) {
        case 4: launch_k(segvec_kernel<F, K, 4>, grid, SEGT_THREADS, 0, st, f, prob, n_seg, skip); break;
        case 8: launch_k(segvec_kernel<F, K, 8>, grid, SEGT_THREADS, 0, st, f, prob, n_seg, skip); break;
        case 16: launch_k(segvec_kernel<F, K, 16>, grid, SEGT_THREADS, 0, st, f, prob, n_seg, skip); break;
        default: launch_k(segvec_kernel<F, K, 32>, grid, SEGT_THREADS, 0, st, f, prob, n_seg, skip); break;
    }
    ++g_launches;
}

template <class F, int K>
void launch_sr(const F& f, const DevPlan& p, uint32_t lo, uint32_t hi, const int* skip, cudaStream_t st) {
    if (hi <= lo) return;
    if (p.ss) {
        constexpr uint32_t WPB = SS_THREADS / 32;
        launch_k(segsweep_kernel<F, K>, (hi - lo + WPB - 1) / WPB, SS_THREADS, 0, st, 
            f, p.ranges, lo, hi, p.bits, p.nz_ids, p.empties, p.ss_splits, p.head, p.tail, p.counters, skip);
        ++g_launches;
        return;
    }
    if constexpr (K <= 2) {
        if (p.wide) {
            launch_k(segreduce_kernel<F, K, sr_items_wide<K>()>, hi - lo, SR_THREADS, 0, st, 
                f, p.tiles, lo, p.splits, p.head, p.tail, p.counters, skip);
            ++g_launches;
            return;
        }
    }
    launch_k(segreduce_kernel<F, K>, hi - lo, SR_THREADS, 0, st, f, p.tiles, lo, p.splits, p.head, p.tail,
                                                           p.counters, skip);
    ++g_launches;
}

int k_bucket(uint64_t k) { return k <= 1 ? 1 : k <= 2 ? 2 : k <= 4 ? 4 : 8; }

// MlsmrOptions extras of one solve (lsmr.rs:155-171): warm start (device,
// column-major n_dofs x k) and the Staleness escalation rule
struct SolveExt {
    const double* x0 = nullptr;
    uint64_t stale_window = 0;
    double stale_threshold = 0.0;
};

}  // namespace

// ---------------------------------------------------------------------------
struct within_design {
    std::vector<std::vector<uint32_t>> levels;
    std::vector<std::vector<double>> slopes;
    std::vector<int> intercept;
    std::vector<std::vector<size_t>> slope_of;   // per effect: indices into slopes
    uint64_t n_obs = 0, n_dofs = 0;
};

// Shared, immutable preconditioner state on the device.
struct within_preconditioner {
    int device = 0;
    int kind = 0;   // 1 additive, 2 diagonal
    uint32_t n = 0;
    Arena arena;
    double* inv_diag = nullptr;
    SchwarzHost host;            // kept for plan building and statistics
    std::vector<double> host_inv_diag;
    SchwarzDev dev_const{};      // pointers into arena (work pointers filled per user)
    // FP32 copies of the factor values (mixed-precision inner solve), built on first use
    SchwarzDevT<float> dev_const_f{};
    float* inv_diag_f = nullptr;
    bool has_f = false;
    // per-step segment problems
    SegProb *p_restrict = nullptr, *p_ct = nullptr, *p_kept = nullptr, *p_dense = nullptr,
            *p_fwd = nullptr, *p_bwd = nullptr, *p_c = nullptr, *p_prolong = nullptr,
            *p_core = nullptr;
    bool has_dense = false, has_core = false;
    uint32_t n_rounds = 0;
    std::mutex mu;
    std::atomic<int> refs{1};
    struct SchwarzUser* standalone = nullptr;   // plans + work of Preconditioner::apply
    ~within_preconditioner();
};

namespace {

int kidx(int K) { return K == 1 ? 0 : K == 2 ? 1 : K == 4 ? 2 : 3; }

// The device image of P.host (set by the caller).
void upload_schwarz_image(within_preconditioner& P) {
    Arena& A = P.arena;
    SchwarzHost& H = P.host;
    SchwarzDev& D = P.dev_const;
    D.n_sub = H.n_sub;
    UploadBatch U;
    U.add(D.loc_ptr, H.loc_ptr);
    U.add(D.n_elim, H.n_elim);
    U.add(D.red_off, H.red_off);
    U.add(D.n_kept, H.n_kept);
    U.add(D.red_n, H.red_n);
    U.add(D.mode, H.mode);
    U.add(D.glob, H.glob);
    U.add(D.scale, H.scale);
    U.add(D.slot_sub, H.slot_sub);
    U.add(D.inv_e, H.inv_e);
    U.add(D.ct_col, H.ct_col);
    U.add(D.ct_val, H.ct_val);
    U.add(D.ct_rowsum, H.ct_rowsum);
    U.add(D.ct_row_slot, H.ct_row_slot);
    U.add(D.ct_row_red, H.ct_row_red);
    U.add(D.elim_slot, H.elim_slot);
    U.add(D.c_col, H.c_col);
    U.add(D.c_val, H.c_val);
    U.add(D.red_sub, H.red_sub);
    U.add(D.dense_row_slot, H.dense_row_slot);
    U.add(D.dense_col, H.dense_col);
    U.add(D.dense_val, H.dense_val);
    U.add(D.dinv, H.dinv);
    U.add(D.fwd_row, H.fwd_row);
    U.add(D.fwd_col, H.fwd_col);
    U.add(D.fwd_val, H.fwd_val);
    U.add(D.bwd_row, H.bwd_row);
    U.add(D.bwd_col, H.bwd_col);
    U.add(D.bwd_val, H.bwd_val);
    U.add(D.dof_slot, H.dof_slot);
    U.add(D.kept_ptr, H.kept_ptr);
    U.add(D.core_row_slot, H.core_row_slot);
    U.add(D.core_col, H.core_col);
    U.add(D.core_val, H.core_val);
    uint32_t* ct_ptr = nullptr;
    U.add(ct_ptr, H.ct_ptr);
    uint32_t* dense_ptr = nullptr;
    U.add(dense_ptr, H.dense_rows_ptr);
    uint32_t* fwd_ptr = nullptr;
    U.add(fwd_ptr, H.fwd_ptr);
    uint32_t* bwd_ptr = nullptr;
    U.add(bwd_ptr, H.bwd_ptr);
    uint32_t* c_ptr = nullptr;
    U.add(c_ptr, H.c_ptr);
    uint32_t* dof_ptr = nullptr;
    U.add(dof_ptr, H.dof_ptr);
    uint32_t* core_ptr = nullptr;
    U.add(core_ptr, H.core_rows_ptr);
    U.commit(A);
    uint32_t* loc_ptr = const_cast<uint32_t*>(D.loc_ptr);
    uint32_t* kept_ptr = const_cast<uint32_t*>(D.kept_ptr);
    auto one = [&](uint32_t* ptr) { return A.upload(std::vector<SegProb>{SegProb{ptr, 0, 0}}); };
    P.p_restrict = one(loc_ptr);
    P.p_ct = one(ct_ptr);
    P.p_kept = one(kept_ptr);
    P.p_dense = one(dense_ptr);
    P.p_c = one(c_ptr);
    P.p_prolong = one(dof_ptr);
    P.p_core = one(core_ptr);
    P.has_dense = H.dense_rows_ptr.size() > 1;
    P.has_core = H.core_rows_ptr.size() > 1;
    P.n_rounds = H.n_rounds;
    std::vector<SegProb> fw, bw;
    for (uint32_t r = 0; r < H.n_rounds; ++r) {
        fw.push_back(SegProb{fwd_ptr + H.fwd_round_ptr[r], H.fwd_round_ptr[r], 0});
        bw.push_back(SegProb{bwd_ptr + H.bwd_round_ptr[r], H.bwd_round_ptr[r], 0});
    }
    P.p_fwd = A.upload(fw);
    P.p_bwd = A.upload(bw);
}

void upload_schwarz(within_preconditioner& P, SchwarzHost&& S) {
    P.host = std::move(S);
    upload_schwarz_image(P);
}

// Schwarz work buffers of one user (solver) for K columns.
template <class T>
struct SchwarzWorkT {
    T *rl = nullptr, *sl = nullptr, *rb = nullptr, *yv = nullptr, *xv = nullptr, *m1 = nullptr, *m2 = nullptr,
      *m3 = nullptr;
};
using SchwarzWork = SchwarzWorkT<double>;

template <class T>
std::vector<T> cast_vec(const std::vector<double>& v) {
    return std::vector<T>(v.begin(), v.end());
}

// FP32 factor values for the mixed-precision inner solve (index arrays shared).
void ensure_precond_f(within_preconditioner& P) {
    std::lock_guard<std::mutex> g(P.mu);
    if (P.has_f) return;
    Arena& A = P.arena;
    if (P.kind == 2) {
        P.inv_diag_f = A.upload(cast_vec<float>(P.host_inv_diag));
    } else {
        const SchwarzHost& H = P.host;
        const SchwarzDev& D = P.dev_const;
        SchwarzDevT<float>& F = P.dev_const_f;
        F.n_sub = D.n_sub;
        F.loc_ptr = D.loc_ptr;
        F.n_elim = D.n_elim;
        F.red_off = D.red_off;
        F.n_kept = D.n_kept;
        F.red_n = D.red_n;
        F.mode = D.mode;
        F.glob = D.glob;
        F.slot_sub = D.slot_sub;
        F.ct_col = D.ct_col;
        F.ct_row_slot = D.ct_row_slot;
        F.ct_row_red = D.ct_row_red;
        F.elim_slot = D.elim_slot;
        F.c_col = D.c_col;
        F.red_sub = D.red_sub;
        F.dense_row_slot = D.dense_row_slot;
        F.dense_col = D.dense_col;
        F.fwd_row = D.fwd_row;
        F.fwd_col = D.fwd_col;
        F.bwd_row = D.bwd_row;
        F.bwd_col = D.bwd_col;
        F.dof_slot = D.dof_slot;
        F.kept_ptr = D.kept_ptr;
        F.core_row_slot = D.core_row_slot;
        F.core_col = D.core_col;
        F.scale = A.upload(cast_vec<float>(H.scale));
        F.inv_e = A.upload(cast_vec<float>(H.inv_e));
        F.ct_val = A.upload(cast_vec<float>(H.ct_val));
        F.ct_rowsum = A.upload(cast_vec<float>(H.ct_rowsum));
        F.c_val = A.upload(cast_vec<float>(H.c_val));
        F.dense_val = A.upload(cast_vec<float>(H.dense_val));
        F.dinv = A.upload(cast_vec<float>(H.dinv));
        F.fwd_val = A.upload(cast_vec<float>(H.fwd_val));
        F.bwd_val = A.upload(cast_vec<float>(H.bwd_val));
        F.core_val = A.upload(cast_vec<float>(H.core_val));
    }
    P.has_f = true;
}

// Everything one user of a (possibly shared) preconditioner mutates: the tile
// plans' partial/counter buffers and the work vectors, per column bucket K.
struct KPlans {
    DevPlan restrict_, ct, kept, dense, fwd, bwd, c, prolong, core;
    // C, the prolongation and each elimination round on one thread per segment
    // when every segment is short: segment counts (0: segmented reduction)
    uint32_t c_thread = 0, prolong_thread = 0;
    int c_lanes = 0;   // C's rows by groups of this many lanes (segvec_kernel), 0 = one thread each
    std::vector<uint32_t> fwd_thread, bwd_thread;
    // rounds [fuse_lo, n_rounds) run as one single-block launch per direction
    // (rounds_fused_kernel) when each has at most RF_MAX_ROWS short rows
    uint32_t fuse_lo = 0, fuse_hi = 0;
    uint32_t* fwd_rows = nullptr;
    uint32_t* bwd_rows = nullptr;
    SchwarzWork w;
    SchwarzWorkT<float> wf;   // mixed-precision inner solve, allocated on first use
    bool ready = false;
};

}  // namespace

struct SchwarzUser {
    Arena arena;
    KPlans kp[4];
    Tuning tuning;
};

within_preconditioner::~within_preconditioner() { delete standalone; }

namespace {

KPlans& schwarz_user_plans(SchwarzUser& U, const within_preconditioner& P, int K) {
    KPlans& kp = U.kp[kidx(K)];
    if (kp.ready) return kp;
    const SchwarzHost& H = P.host;
    Arena& A = U.arena;
    const int T = plan_tile(K, false);
    const bool ss = U.tuning.warp_ranges >= 2;
    auto one = [&](const std::vector<uint32_t>& ptr, bool ss_plan) {
        const uint32_t n_seg = (uint32_t)ptr.size() - 1;
        if (ss_plan) {
            SSHostPlan sp;
            sp.add(0, ptr.data(), n_seg, ss_range_len(n_seg ? ptr[n_seg] - ptr[0] : 0, ss_target_warps(K)));
            DevPlan d = make_ss_plan(A, sp, K);
            d.range_lo = {0};
            d.range_hi = {d.n_tiles};
            return d;
        }
        HostPlan hp;
        const bool wide = plan_wide(K, n_seg ? ptr[n_seg] - ptr[0] : 0, n_seg, U.tuning.wide_mean_len);
        hp.add(0, ptr.data(), n_seg, plan_tile(K, wide));
        DevPlan d = make_plan(A, hp, K);
        d.wide = wide;
        d.range_lo = {0};
        d.range_hi = {d.n_tiles};
        return d;
    };
    kp.restrict_ = one(H.loc_ptr, ss);
    kp.ct = one(H.ct_ptr, U.tuning.warp_ranges >= 2 || (U.tuning.warp_ranges == 1 && K == 1));
    kp.kept = one(H.kept_ptr, ss);
    kp.dense = one(H.dense_rows_ptr, ss);
    const bool segt_on = U.tuning.segthread;
    if (segt_on && H.c_ptr.size() > 1 && seg_max_len(H.c_ptr.data(), H.c_ptr.size() - 1) <= SEGT_MAX_LEN)
        kp.c_thread = (uint32_t)(H.c_ptr.size() - 1);
    if (kp.c_thread && U.tuning.vector_rows)
        kp.c_lanes = segvec_lanes((double)(H.c_ptr.back() - H.c_ptr.front()) / (double)kp.c_thread);
    if (segt_on && H.dof_ptr.size() > 1 && seg_max_len(H.dof_ptr.data(), H.dof_ptr.size() - 1) <= SEGT_MAX_LEN)
        kp.prolong_thread = (uint32_t)(H.dof_ptr.size() - 1);
    // tile plans only where the one-thread-per-segment kernels are not used
    if (!kp.c_thread) kp.c = one(H.c_ptr, ss);
    if (!kp.prolong_thread) kp.prolong = one(H.dof_ptr, ss);
    kp.core = one(H.core_rows_ptr, ss);
    auto rounds = [&](const std::vector<uint32_t>& rptr, const std::vector<uint32_t>& ptr) {
        if (ss) {
            SSHostPlan sp;
            std::vector<uint32_t> lo, hi;
            for (uint32_t r = 0; r + 1 < rptr.size(); ++r) {
                const uint32_t* rp = ptr.data() + rptr[r];
                const uint32_t m = rptr[r + 1] - rptr[r];
                lo.push_back((uint32_t)sp.ranges.size());
                sp.add(r, rp, m, ss_range_len(m ? rp[m] - rp[0] : 0, ss_target_warps(K)));
                hi.push_back((uint32_t)sp.ranges.size());
            }
            DevPlan d = make_ss_plan(A, sp, K);
            d.range_lo = lo;
            d.range_hi = hi;
            return d;
        }
        HostPlan hp;
        std::vector<uint32_t> lo, hi;
        for (uint32_t r = 0; r + 1 < rptr.size(); ++r) {
            lo.push_back((uint32_t)hp.tiles.size());
            hp.add(r, ptr.data() + rptr[r], rptr[r + 1] - rptr[r], T);
            hi.push_back((uint32_t)hp.tiles.size());
        }
        DevPlan d = make_plan(A, hp, K);
        d.range_lo = lo;
        d.range_hi = hi;
        return d;
    };
    kp.fwd = rounds(H.fwd_round_ptr, H.fwd_ptr);
    kp.bwd = rounds(H.bwd_round_ptr, H.bwd_ptr);
    auto round_thread = [&](const std::vector<uint32_t>& rptr, const std::vector<uint32_t>& ptr) {
        std::vector<uint32_t> nseg;
        for (size_t r = 0; r + 1 < rptr.size(); ++r) {
            const uint32_t m = rptr[r + 1] - rptr[r];
            nseg.push_back(segt_on && m && seg_max_len(ptr.data() + rptr[r], m) <= SEGT_MAX_LEN ? m : 0u);
        }
        return nseg;
    };
    kp.fwd_thread = round_thread(H.fwd_round_ptr, H.fwd_ptr);
    kp.bwd_thread = round_thread(H.bwd_round_ptr, H.bwd_ptr);
    // the fused tail: the longest suffix of rounds that are one-thread rounds
    // in both directions with at most RF_MAX_ROWS rows (WITHIN_FUSE_ROUNDS=0: none)
    {
        const bool fuse_on = segt_on && U.tuning.fuse_rounds;
        const uint32_t nr = H.n_rounds;
        uint32_t lo = nr;
        auto ok = [&](uint32_t r) {
            const uint32_t fr = H.fwd_round_ptr[r + 1] - H.fwd_round_ptr[r];
            const uint32_t br = H.bwd_round_ptr[r + 1] - H.bwd_round_ptr[r];
            return (fr == 0 || kp.fwd_thread[r]) && (br == 0 || kp.bwd_thread[r]) && fr <= RF_MAX_ROWS &&
                   br <= RF_MAX_ROWS;
        };
        while (fuse_on && lo > 0 && ok(lo - 1)) --lo;
        if (nr - lo >= 2) {
            kp.fuse_lo = lo;
            kp.fuse_hi = nr;
            std::vector<uint32_t> fr(nr), br(nr);
            for (uint32_t r = 0; r < nr; ++r) {
                fr[r] = H.fwd_round_ptr[r + 1] - H.fwd_round_ptr[r];
                br[r] = H.bwd_round_ptr[r + 1] - H.bwd_round_ptr[r];
            }
            kp.fwd_rows = A.upload(fr);
            kp.bwd_rows = A.upload(br);
        }
    }
    size_t nl = H.glob.size(), nr = H.n_red, ns = H.n_sub;
    kp.w.rl = A.alloc<double>(nl * K);
    kp.w.sl = A.alloc<double>(nl * K);
    kp.w.rb = A.alloc<double>(nr * K);
    kp.w.yv = A.alloc<double>(nr * K);
    kp.w.xv = A.alloc<double>(nr * K);
    kp.w.m1 = A.alloc<double>(ns * K);
    kp.w.m2 = A.alloc<double>(ns * K);
    kp.w.m3 = A.alloc<double>(ns * K);
    kp.ready = true;
    return kp;
}

// FP32 work vectors of one user (allocated outside any stream capture).
SchwarzWorkT<float>& schwarz_user_work_f(SchwarzUser& U, const within_preconditioner& P, int K) {
    KPlans& kp = schwarz_user_plans(U, P, K);
    if (!kp.wf.rl) {
        const SchwarzHost& H = P.host;
        size_t nl = H.glob.size(), nr = H.n_red, ns = H.n_sub;
        kp.wf.rl = U.arena.alloc<float>(nl * K);
        kp.wf.sl = U.arena.alloc<float>(nl * K);
        kp.wf.rb = U.arena.alloc<float>(nr * K);
        kp.wf.yv = U.arena.alloc<float>(nr * K);
        kp.wf.xv = U.arena.alloc<float>(nr * K);
        kp.wf.m1 = U.arena.alloc<float>(ns * K);
        kp.wf.m2 = U.arena.alloc<float>(ns * K);
        kp.wf.m3 = U.arena.alloc<float>(ns * K);
    }
    return kp.wf;
}

template <int K, class T = double>
void schwarz_apply(within_preconditioner& P, SchwarzUser& U, const T* r, T* z, const int* skip,
                   cudaStream_t st) {
    KPlans& kp = schwarz_user_plans(U, P, K);
    SchwarzDevT<T> S;
    SchwarzWorkT<T>* w;
    if constexpr (sizeof(T) == 8) {
        S = P.dev_const;
        w = &kp.w;
    } else {
        S = P.dev_const_f;
        w = &schwarz_user_work_f(U, P, K);
    }
    S.rl = w->rl;
    S.sl = w->sl;
    S.rb = w->rb;
    S.yv = w->yv;
    S.xv = w->xv;
    S.m1 = w->m1;
    S.m2 = w->m2;
    S.m3 = w->m3;
    using RF = RestrictF<K, T>;
    using CtFT = CtF<K, T>;
    using KS = KeptSumF<K, T>;
    using DF = DenseF<K, T>;
    using FF = FwdF<K, T>;
    using CoF = CoreF<K, T>;
    using BF = BwdF<K, T>;
    using CFT = CF<K, T>;
    using MF = MeanF<K, T>;
    using PF = ProlongF<K, T>;
    launch_sr<RF, K>(RF{P.p_restrict, S, r}, kp.restrict_, 0, kp.restrict_.n_tiles, skip, st);
    launch_sr<CtFT, K>(CtFT{P.p_ct, S}, kp.ct, 0, kp.ct.n_tiles, skip, st);
    launch_sr<KS, K>(KS{P.p_kept, S}, kp.kept, 0, kp.kept.n_tiles, skip, st);
    if (P.has_dense) launch_sr<DF, K>(DF{P.p_dense, S}, kp.dense, 0, kp.dense.n_tiles, skip, st);
    const bool fused = kp.fuse_hi > kp.fuse_lo;
    const uint32_t r_fwd_end = fused ? kp.fuse_lo : P.n_rounds;
    for (uint32_t r = 0; r < r_fwd_end; ++r) {
        if (kp.fwd_thread[r]) launch_segthread<FF, K>(FF{P.p_fwd, S}, r, kp.fwd_thread[r], skip, st);
        else launch_sr<FF, K>(FF{P.p_fwd, S}, kp.fwd, kp.fwd.range_lo[r], kp.fwd.range_hi[r], skip, st);
    }
    if (fused) {
        launch_k(rounds_fused_kernel<FF, K>, 1, RF_THREADS, 0, st, FF{P.p_fwd, S}, kp.fwd_rows, kp.fuse_lo, kp.fuse_hi, 0,
                                                              skip);
        ++g_launches;
    }
    if (P.has_core) launch_sr<CoF, K>(CoF{P.p_core, S}, kp.core, 0, kp.core.n_tiles, skip, st);
    if (fused) {
        launch_k(rounds_fused_kernel<BF, K>, 1, RF_THREADS, 0, st, BF{P.p_bwd, S}, kp.bwd_rows, kp.fuse_lo, kp.fuse_hi, 1,
                                                              skip);
        ++g_launches;
    }
    for (uint32_t r = r_fwd_end; r-- > 0;) {
        if (kp.bwd_thread[r]) launch_segthread<BF, K>(BF{P.p_bwd, S}, r, kp.bwd_thread[r], skip, st);
        else launch_sr<BF, K>(BF{P.p_bwd, S}, kp.bwd, kp.bwd.range_lo[r], kp.bwd.range_hi[r], skip, st);
    }
    if (kp.c_thread && kp.c_lanes) launch_segvec<CFT, K>(CFT{P.p_c, S}, 0, kp.c_thread, kp.c_lanes, skip, st);
    else if (kp.c_thread) launch_segthread<CFT, K>(CFT{P.p_c, S}, 0, kp.c_thread, skip, st);
    else launch_sr<CFT, K>(CFT{P.p_c, S}, kp.c, 0, kp.c.n_tiles, skip, st);
    launch_sr<MF, K>(MF{P.p_restrict, S}, kp.restrict_, 0, kp.restrict_.n_tiles, skip, st);
    if (kp.prolong_thread) launch_segthread<PF, K>(PF{P.p_prolong, S, z}, 0, kp.prolong_thread, skip, st);
    else launch_sr<PF, K>(PF{P.p_prolong, S, z}, kp.prolong, 0, kp.prolong.n_tiles, skip, st);
}

}  // namespace

// ---------------------------------------------------------------------------
struct within_solver {
    int device = 0;
    cudaStream_t stream = nullptr;
    HostDesign design;
    Reparam reparam;
    uint64_t n_obs = 0, n_dofs = 0;
    uint64_t n_warnings = 0;
    within_preconditioner* precond = nullptr;
    int precision = WITHIN_PRECISION_FP64;
    std::mutex mu;
    Arena arena;
    // design on device
    OpParams op{};
    uint32_t* perm = nullptr;               // internal -> caller (nullptr = identity)
    std::vector<ScatterProb> scatter_host;  // problems (same for all K)
    ScatterProb* scatter_probs = nullptr;
    // mixed precision: FP32 copies of sqrt(w) and the loading columns
    OpParamsT<float> op_f{};
    ScatterProb* scatter_probs_f = nullptr;
    bool has_f = false;
    std::vector<std::vector<uint32_t>> level_ptr_host;   // per term
    DevPlan scatter_plan[4];
    bool scatter_ready[4] = {false, false, false, false};
    // workspaces per K
    struct Work {
        bool ready = false;
        bool buffers = false;   // the vectors below are allocated
        double *u, *b, *yint, *v, *p, *h, *hb, *x, *dm;
        double* x0 = nullptr;   // warm start, interleaved (allocated on first use)
        double* partials;
        unsigned* counter;
        double* bmax;
        int* nonfinite;
        ColState* st;   // [2][K]
        Ctl* ctl;
        cudaGraphExec_t graph = nullptr;       // two iterations, replayed in bursts
        uint64_t graph_iters = 0;
        cudaGraphExec_t loop_graph = nullptr;  // the whole loop: a device-side while node
        bool loop_failed = false;
        // windowed reorthogonalisation (local_size): the ring the graphs were built for
        Ring ring{nullptr, nullptr, 0};
        double* coef = nullptr;
        uint64_t ring_alloc = 0;   // slots allocated
    } work[4];
    // mixed-precision workspaces per K (refine.cuh)
    struct MixedWork {
        bool ready = false;
        double *r64, *g64, *x64;
        float *res, *z, *p, *q, *t, *d;
        CgCol* st;
        Ctl* ctl;
        cudaGraphExec_t loop_graph = nullptr;
        uint64_t body_launches = 0;
        cudaGraphExec_t solve_graph = nullptr;   // refinement steps and inner loops, all on the device
        bool solve_graph_failed = false;
        uint64_t pre_launches = 0, post_launches = 0;
    } mixed[4];
    // pinned staging for the host entry points
    double* pin = nullptr;
    size_t pin_n = 0;
    SchwarzUser schwarz;   // this solver's plans/work for the preconditioner
    // warp-range row sweep (rowsweep.cuh), per column bucket K
    struct RowSweepK {
        bool ready = false;
        RwParams rp{};
        size_t smem = 0;
        std::vector<ScatterProb> rest_host;   // run combines + full-resolution rest terms
        std::vector<std::vector<uint32_t>> rest_ptrs;
        DevPlan rest;
        ScatterProb* rest_probs = nullptr;
        ScatterProb* rest_probs_f = nullptr;
        uint32_t n_rest = 0;
        bool rest_needs_rows = false;        // a full-resolution rest term reads the row vector
        bool simple = false;                 // every term intercept-only: the specialised sweep
        double* atu = nullptr;               // n_dofs * K raw A^T u (LSMR)
        size_t smem_f = 0;                   // shared memory of the FP32 normal-operator mode
        int grid = 0;                        // blocks of every sweep launch (the ranges are cut for it)
        // staged sweep (tsweep.cuh): used for the FP64 adjoint and LSMR-step modes
        bool ts = false;
        TsSlots ts_slots{};
        int ts_nq = 0;
        size_t ts_smem = 0;
    } rsw[4];
    int* sweep_err = nullptr;   // device flag of a timed-out wait in a sweep outside the LSMR loop
    // per column bucket, the LSMR step's operator path:
    // 0 gather + full segmented-reduction scatter, 2 warp-range row sweep (rowsweep.cuh)
    int path[4] = {0, 0, 0, 0};

    ~within_solver() {
        for (auto& w : work) {
            if (w.graph) cudaGraphExecDestroy(w.graph);
            if (w.loop_graph) cudaGraphExecDestroy(w.loop_graph);
        }
        for (auto& m : mixed) {
            if (m.loop_graph) cudaGraphExecDestroy(m.loop_graph);
            if (m.solve_graph) cudaGraphExecDestroy(m.solve_graph);
        }
        if (pin) cudaFreeHost(pin);
        if (stream) cudaStreamDestroy(stream);
        if (precond && --precond->refs == 0) delete precond;
    }
};

namespace {

constexpr int RED_GRID = 148 * 8;    // fixed reduction grid: deterministic partial order

void set_device(int dev) { CK(cudaSetDevice(dev)); }

// Integer passes over a column of codes on the host pool (chunks of 2^20
// observations; every result is an exact count, so it does not depend on the
// schedule).
constexpr uint64_t CODE_CHUNK = (uint64_t)1 << 20;

// number of runs (maximal blocks of equal consecutive codes)
uint64_t count_runs(const uint32_t* codes, uint64_t n) {
    const size_t nch = (size_t)((n + CODE_CHUNK - 1) / CODE_CHUNK);
    std::vector<uint64_t> part(nch, 0);
    par_for_each(nch, [&](size_t c) {
        const uint64_t i0 = c * CODE_CHUNK, i1 = std::min(n, i0 + CODE_CHUNK);
        uint64_t r = 0;
        for (uint64_t i = i0; i < i1; ++i) r += (i == 0 || codes[i] != codes[i - 1]) ? 1 : 0;
        part[c] = r;
    });
    uint64_t runs = 0;
    for (uint64_t r : part) runs += r;
    return runs;
}

// the level of every run, in run order
std::vector<uint32_t> run_levels(const uint32_t* codes, uint64_t n, uint64_t runs) {
    const size_t nch = (size_t)((n + CODE_CHUNK - 1) / CODE_CHUNK);
    std::vector<uint64_t> off(nch + 1, 0);
    par_for_each(nch, [&](size_t c) {
        const uint64_t i0 = c * CODE_CHUNK, i1 = std::min(n, i0 + CODE_CHUNK);
        uint64_t r = 0;
        for (uint64_t i = i0; i < i1; ++i) r += (i == 0 || codes[i] != codes[i - 1]) ? 1 : 0;
        off[c + 1] = r;
    });
    for (size_t c = 0; c < nch; ++c) off[c + 1] += off[c];
    std::vector<uint32_t> lv(runs);
    par_for_each(nch, [&](size_t c) {
        const uint64_t i0 = c * CODE_CHUNK, i1 = std::min(n, i0 + CODE_CHUNK);
        uint64_t q = off[c];
        for (uint64_t i = i0; i < i1; ++i)
            if (i == 0 || codes[i] != codes[i - 1]) lv[q++] = codes[i];
    });
    return lv;
}

// lp[l] = number of codes below l (lp has n_levels + 1 entries)
void level_counts(const uint32_t* codes, uint64_t n, uint32_t n_levels, std::vector<uint32_t>& lp) {
    lp.assign((size_t)n_levels + 1, 0);
    const size_t nch = (size_t)std::min<uint64_t>(16, (n + CODE_CHUNK - 1) / CODE_CHUNK);
    if (nch <= 1 || (uint64_t)n_levels * nch > ((uint64_t)1 << 24)) {
        for (uint64_t i = 0; i < n; ++i) ++lp[(size_t)codes[i] + 1];
    } else {
        const uint64_t per = (n + nch - 1) / nch;
        std::vector<std::vector<uint32_t>> h(nch);
        par_for_each(nch, [&](size_t c) {
            h[c].assign((size_t)n_levels + 1, 0);
            const uint64_t i0 = c * per, i1 = std::min(n, i0 + per);
            for (uint64_t i = i0; i < i1; ++i) ++h[c][(size_t)codes[i] + 1];
        });
        const size_t B = 65536;
        par_for_each(((size_t)n_levels + 1 + B - 1) / B, [&](size_t b) {
            const size_t l1 = std::min<size_t>((size_t)n_levels + 1, (b + 1) * B);
            for (size_t l = b * B; l < l1; ++l) {
                uint32_t t = 0;
                for (size_t c = 0; c < nch; ++c) t += h[c][l];
                lp[l] = t;
            }
        });
    }
    for (uint32_t l = 0; l < n_levels; ++l) lp[l + 1] += lp[l];
}

void ensure_scatter(within_solver& s, int K) {
    int ki = kidx(K);
    if (s.scatter_ready[ki]) return;
    const int T = K == 1 ? sr_tile<1>() : K == 2 ? sr_tile<2>() : K == 4 ? sr_tile<4>() : sr_tile<8>();
    HostPlan hp;
    uint32_t prob = 0;
    for (size_t t = 0; t < s.design.terms.size(); ++t) {
        const auto& lp = s.level_ptr_host[t];
        for (size_t c = 0; c < s.design.terms[t].cols.size(); ++c)
            hp.add(prob++, lp.data(), (uint32_t)lp.size() - 1, T);
    }
    s.scatter_plan[ki] = make_plan(s.arena, hp, K);
    s.scatter_ready[ki] = true;
}

// The staged sweep instantiations (K = 1): mode 0 (adjoint) and 1 (LSMR
// step) for every class layout of at most three terms; nullptr when the
// layout has none.
using TsKernel = void (*)(OpParams, RwParams, TsSlots, const double*, double*, ColState*, Ctl*, int*);
template <int MODE, int NQ, int NRUN, int NHIST, bool WTD>
TsKernel ts_pick() {
    if constexpr (NRUN + NHIST <= NQ) return k_tsweep<1, MODE, NQ, NRUN, NHIST, WTD>;
    else return nullptr;
}
template <int MODE, int NQ, int NRUN, bool WTD>
TsKernel ts_pick_h(int nhist) {
    switch (nhist) {
        case 0: return ts_pick<MODE, NQ, NRUN, 0, WTD>();
        case 1: return ts_pick<MODE, NQ, NRUN, 1, WTD>();
        default: return ts_pick<MODE, NQ, NRUN, 2, WTD>();
    }
}
template <int MODE, int NQ, bool WTD>
TsKernel ts_pick_r(int nrun, int nhist) {
    return nrun == 1 ? ts_pick_h<MODE, NQ, 1, WTD>(nhist) : ts_pick_h<MODE, NQ, 2, WTD>(nhist);
}
template <int MODE, bool WTD>
TsKernel ts_pick_q(int nq, int nrun, int nhist) {
    switch (nq) {
        case 1: return ts_pick_r<MODE, 1, WTD>(nrun, nhist);
        case 2: return ts_pick_r<MODE, 2, WTD>(nrun, nhist);
        default: return ts_pick_r<MODE, 3, WTD>(nrun, nhist);
    }
}
TsKernel ts_kernel(int mode, int nq, int nrun, int nhist, bool wtd) {
    if (nq < 1 || nq > TS_MAXQ || nrun < 1 || nrun > RW_MAX_RUN || nhist < 0 || nhist > RW_MAX_HIST) return nullptr;
    if (mode == 0) return wtd ? ts_pick_q<0, true>(nq, nrun, nhist) : ts_pick_q<0, false>(nq, nrun, nhist);
    return wtd ? ts_pick_q<1, true>(nq, nrun, nhist) : ts_pick_q<1, false>(nq, nrun, nhist);
}

// The staged gather / demeaning instantiations (K = 1, intercept-only, at
// most three terms); nullptr outside them.
using TgKernel = void (*)(OpParams, const double*, const double*, double*, const int*, int*);
template <bool WTD, bool DEMEAN>
TgKernel tg_pick(int nq) {
    switch (nq) {
        case 1: return k_tgather<1, WTD, DEMEAN>;
        case 2: return k_tgather<2, WTD, DEMEAN>;
        case 3: return k_tgather<3, WTD, DEMEAN>;
        default: return nullptr;
    }
}
TgKernel tg_kernel(int nq, bool wtd, bool demean) {
    if (demean) return tg_pick<false, true>(nq);
    return wtd ? tg_pick<true, false>(nq) : tg_pick<false, false>(nq);
}
size_t tg_smem(int nq, bool wtd, bool demean) {
    const size_t stage = (size_t)TG_CH * (4 * nq + (demean ? 8 : 0) + (wtd && !demean ? 8 : 0));
    return (size_t)RW_WARPS * TS_STAGES * (stage + sizeof(uint64_t));
}
// whether the staged gather applies to this solver's design (WITHIN_TSWEEP=0: never)
bool tg_applies(const within_solver& s) {
    if (!s.schwarz.tuning.staged) return false;
    if (s.design.terms.size() > (size_t)TS_MAXQ || s.design.terms.empty()) return false;
    for (const Term& T : s.design.terms)
        if (T.cols.size() != 1 || T.cols[0] >= 0) return false;
    return true;
}
// y = W^{1/2} D x (demean: out = yint - D x) through the staged gather when it
// applies and the output is 16-byte aligned; returns false otherwise
bool launch_tgather(within_solver& s, const double* x, const double* yint, double* out, bool demean,
                    const int* skip, int* err, cudaStream_t st) {
    if (!tg_applies(s) || ((uintptr_t)out & 15) != 0) return false;
    const int nq = (int)s.design.terms.size();
    const bool wtd = s.op.sqrt_w != nullptr && !demean;
    TgKernel f = tg_kernel(nq, wtd, demean);
    if (!f) return false;
    const size_t sm = tg_smem(nq, wtd, demean);
    {
        static std::mutex mu;
        static std::vector<std::pair<int, TgKernel>> done;
        std::lock_guard<std::mutex> g(mu);
        int dev = 0;
        CK(cudaGetDevice(&dev));
        if (std::find(done.begin(), done.end(), std::make_pair(dev, f)) == done.end()) {
            CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tg_smem(3, true, true)));
            done.emplace_back(dev, f);
        }
    }
    launch_k(f, TG_GRID, RW_THREADS, sm, st, s.op, x, yint, out, skip, err);
    ++g_launches;
    return true;
}

// Classifies the terms for the warp-range row sweep and builds its tables
// (rowsweep.cuh): range bases of the run ordinals, the crossing-run fix-ups,
// the level-sorted run combines and the remaining full-resolution terms.
template <int K>
within_solver::RowSweepK& ensure_rowsweep(within_solver& s) {
    auto& rk = s.rsw[kidx(K)];
    if (rk.ready) return rk;
    const HostDesign& D = s.design;
    const uint64_t n = D.n_obs;
    Arena& A = s.arena;
    RwParams& rp = rk.rp;
    const int Q = (int)D.terms.size();
    // term classes: hist (few coefficients), run (sorted, or few runs), rest
    enum { CLS_REST = 0, CLS_RUN = 1, CLS_HIST = 2 };
    std::vector<int> cls(Q, CLS_REST);
    std::vector<uint64_t> n_runs(Q, 0);
    {
        int nh = 0, nr = 0, nbk = 0;
        for (int t = 0; t < Q; ++t) {
            const Term& T = D.terms[t];
            const auto& codes = D.codes[t];
            const int ncol = (int)T.cols.size();
            if (nh < RW_MAX_HIST && (uint64_t)nbk + (uint64_t)T.n_levels * ncol <= RW_MAX_BUCKETS) {
                cls[t] = CLS_HIST;
                ++nh;
                nbk += (int)(T.n_levels * ncol);
                continue;
            }
            const uint64_t runs = count_runs(codes.data(), n);
            n_runs[t] = runs;
            if (nr < RW_MAX_RUN && ncol <= rw_max_cols<K>() && (T.sorted != 0 || runs * 3 <= n)) {
                cls[t] = CLS_RUN;
                ++nr;
            }
        }
    }
    bool simple = true;
    for (const Term& T : D.terms)
        if (T.cols.size() != 1 || T.cols[0] >= 0) simple = false;
    // the staged sweep: intercept-only, at most three terms, one run term or
    // more, its shared memory within two blocks per SM (WITHIN_TSWEEP=0: never)
    {
        int nrun = 0, nhist = 0, nbk = 0;
        for (int t = 0; t < Q; ++t) {
            nrun += cls[t] == CLS_RUN;
            nhist += cls[t] == CLS_HIST;
            if (cls[t] == CLS_HIST) nbk += (int)D.terms[t].n_levels;
        }
        const bool ok = K == 1 && simple && Q <= TS_MAXQ && nrun >= 1 && s.schwarz.tuning.staged;
        const size_t sm = ts_smem_bytes<K>(nbk, nhist, Q, s.op.sqrt_w != nullptr);
        if (ok && sm <= TS_SMEM_CAP) {
            rk.ts = true;
            rk.ts_nq = Q;
            rk.ts_smem = sm;
            int k = 0;
            for (int t = 0; t < Q; ++t)
                if (cls[t] == CLS_RUN) rk.ts_slots.term[k++] = t;
            for (int t = 0; t < Q; ++t)
                if (cls[t] == CLS_HIST) rk.ts_slots.term[k++] = t;
            for (int t = 0; t < Q; ++t)
                if (cls[t] == CLS_REST) rk.ts_slots.term[k++] = t;
        }
    }
    rk.grid = rk.ts ? TS_GRID : rw_grid<K>();
    const uint64_t G = (uint64_t)rk.grid * RW_WARPS;
    const uint64_t CH = rw_chunk<K>();
    uint64_t rpr = (n + G - 1) / G;
    rpr = std::max<uint64_t>(CH, (rpr + CH - 1) / CH * CH);
    rp.rows_per_range = (uint32_t)rpr;
    std::vector<RwFix> fixes;
    size_t first_prob = 0;
    for (int t = 0; t < Q; ++t) {
        const Term& T = D.terms[t];
        const auto& codes = D.codes[t];
        const int ncol = (int)T.cols.size();
        const size_t probs_before = first_prob;
        first_prob += (size_t)ncol;
        if (cls[t] == CLS_HIST) {
            rp.hist[rp.n_hist++] = RwHist{t, rp.n_buckets};
            rp.n_buckets += (int)(T.n_levels * ncol);
            continue;
        }
        if (cls[t] == CLS_RUN) {
            // run heads per range
            std::vector<uint32_t> cnt(G, 0);
            const uint64_t runs = n_runs[t];
            par_for_each((size_t)((G + 63) / 64), [&](size_t b) {
                for (uint64_t g = b * 64; g < std::min<uint64_t>(G, (b + 1) * 64); ++g) {
                    const uint64_t i0 = g * rpr, i1 = std::min<uint64_t>(n, i0 + rpr);
                    uint32_t c = 0;
                    for (uint64_t i = i0; i < i1; ++i) c += (i == 0 || codes[i] != codes[i - 1]) ? 1u : 0u;
                    cnt[g] = c;
                }
            });
            const bool sorted_runs = T.sorted != 0;
            const int j = rp.n_run++;
            RwRun& rr = rp.run[j];
            rr.term = t;
            rr.direct = sorted_runs ? 1 : 0;
            std::vector<uint32_t> base(G, 0);
            for (uint64_t g = 1; g < G; ++g) base[g] = base[g - 1] + cnt[g - 1];
            for (uint64_t g = 0; g < G; ++g) {
                const uint64_t r0 = g * rpr, r1 = std::min<uint64_t>(r0 + rpr, n);
                if (r0 >= n) break;
                if (cnt[g] == 0 || r1 >= n || codes[r1] != codes[r1 - 1]) continue;
                uint64_t h = g + 1;
                while (true) {
                    const uint64_t h0 = h * rpr, h1 = std::min<uint64_t>(h0 + rpr, n);
                    if (cnt[h] > 0 || h1 >= n || codes[h1] != codes[h1 - 1]) break;
                    (void)h0;
                    ++h;
                }
                RwFix f;
                f.g0 = (uint32_t)g;
                f.g1 = (uint32_t)h;
                f.id = rr.direct ? codes[r1 - 1] : base[g] + cnt[g] - 1;
                f.run = (uint32_t)j;
                fixes.push_back(f);
            }
            rr.head = A.alloc<double>(G * ncol * K);
            rr.tail = A.alloc<double>(G * ncol * K);
            rr.range_base = nullptr;
            rr.run_sum = nullptr;
            if (!rr.direct) {
                rr.range_base = A.upload(base);
                rr.run_sum = A.alloc<double>(runs * ncol * K);
                // combine: run sums grouped by level (stable in run order)
                std::vector<uint32_t> run_level = run_levels(codes.data(), n, runs);
                std::vector<uint32_t> perm(runs);
                stable_argsort_u32(run_level.data(), runs, T.n_levels, perm.data());
                std::vector<uint32_t> lp((size_t)T.n_levels + 1, 0);
                for (uint32_t l : run_level) ++lp[(size_t)l + 1];
                for (uint32_t l = 0; l < T.n_levels; ++l) lp[l + 1] += lp[l];
                uint32_t* dlp = A.upload(lp);
                uint32_t* dperm = A.upload(perm);
                for (int c = 0; c < ncol; ++c) {
                    ScatterProb pr{};
                    pr.seg_ptr = dlp;
                    pr.order = dperm;
                    pr.out_off = (uint32_t)(T.offset + c * T.n_levels);
                    pr.ncol = (uint32_t)ncol;
                    pr.run_sum = rr.run_sum;
                    pr.col = (uint32_t)c;
                    rk.rest_host.push_back(pr);
                    rk.rest_ptrs.push_back(lp);
                }
            }
            continue;
        }
        for (int c = 0; c < ncol; ++c) {
            rk.rest_host.push_back(s.scatter_host[probs_before + c]);
            rk.rest_ptrs.push_back(s.level_ptr_host[t]);
            rk.rest_needs_rows = true;
        }
    }
    rp.fix = A.upload(fixes);
    rp.n_fix = (uint32_t)fixes.size();
    rk.simple = true;
    for (const Term& T : D.terms)
        if (T.cols.size() != 1 || T.cols[0] >= 0) rk.simple = false;
    rp.part = A.alloc<double>((size_t)rk.grid * (K + (size_t)rp.n_buckets * K));
    rp.counter = A.alloc<unsigned>(1);
    // histogram shared memory per bin type (FP64 modes / the FP32 normal operator)
    bool pv;
    rk.smem = rw_smem_bytes<K, 8>(rp.n_buckets, rp.n_hist, pv);
    rk.smem_f = rw_smem_bytes<K, 4>(rp.n_buckets, rp.n_hist, pv);
    rk.atu = A.alloc<double>(s.n_dofs * K);
    rk.n_rest = (uint32_t)rk.rest_host.size();
    if (rk.n_rest) {
        uint64_t pos = 0, segs = 0;
        for (const auto& lp : rk.rest_ptrs) {
            pos += lp.back() - lp.front();
            segs += lp.size() - 1;
        }
        if (s.schwarz.tuning.warp_ranges >= 2 || (s.schwarz.tuning.warp_ranges == 1 && K == 1)) {
            SSHostPlan sp;
            const uint32_t L = ss_range_len(pos, ss_target_warps(K));
            for (size_t i = 0; i < rk.rest_host.size(); ++i)
                sp.add((uint32_t)i, rk.rest_ptrs[i].data(), (uint32_t)rk.rest_ptrs[i].size() - 1, L);
            rk.rest = make_ss_plan(A, sp, K);
        } else {
            const bool wide = plan_wide(K, pos, segs, s.schwarz.tuning.wide_mean_len);
            const int Ttile = plan_tile(K, wide);
            HostPlan hp;
            for (size_t i = 0; i < rk.rest_host.size(); ++i)
                hp.add((uint32_t)i, rk.rest_ptrs[i].data(), (uint32_t)rk.rest_ptrs[i].size() - 1, Ttile);
            rk.rest = make_plan(A, hp, K);
            rk.rest.wide = wide;
        }
        rk.rest_probs = A.upload(rk.rest_host);
    }
    // dynamic shared memory above the default needs the opt-in (set outside any capture)
    // The dynamic shared-memory ceiling is a property of the kernel function
    // (shared by every solver in the process), so it is raised once per device
    // to a bound that covers every design, never to one design's size.
    {
        static std::mutex mu;
        static std::vector<std::pair<int, int>> done;
        std::lock_guard<std::mutex> g(mu);
        int dev = 0;
        CK(cudaGetDevice(&dev));
        if (std::find(done.begin(), done.end(), std::make_pair(dev, K)) == done.end()) {
            const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
            const int cap = (int)RW_SMEM_CAP;
            CK(cudaFuncSetAttribute(k_rowsweep<K, 0, double, false>, attr, cap));
            CK(cudaFuncSetAttribute(k_rowsweep<K, 1, double, false>, attr, cap));
            CK(cudaFuncSetAttribute(k_rowsweep<K, 2, float, false>, attr, cap));
            CK(cudaFuncSetAttribute(k_rowsweep<K, 3, double, false>, attr, cap));
            CK(cudaFuncSetAttribute(k_rowsweep<K, 0, double, true>, attr, cap));
            CK(cudaFuncSetAttribute(k_rowsweep<K, 1, double, true>, attr, cap));
            CK(cudaFuncSetAttribute(k_rowsweep<K, 2, float, true>, attr, cap));
            CK(cudaFuncSetAttribute(k_rowsweep<K, 3, double, true>, attr, cap));
            if constexpr (K == 1) {
                for (int mode = 0; mode < 2; ++mode)
                    for (int nq = 1; nq <= TS_MAXQ; ++nq)
                        for (int nrun = 1; nrun <= RW_MAX_RUN; ++nrun)
                            for (int nhist = 0; nhist <= RW_MAX_HIST; ++nhist)
                                for (int wtd = 0; wtd < 2; ++wtd)
                                    if (auto f = ts_kernel(mode, nq, nrun, nhist, wtd != 0))
                                        CK(cudaFuncSetAttribute(f, attr, (int)TS_SMEM_CAP));
            }
            done.emplace_back(dev, K);
        }
    }
    rk.ready = true;
    return rk;
}

// FP32 loading columns in the rest problems (mixed-precision inner solve)
template <int K>
void ensure_rowsweep_f(within_solver& s) {
    auto& rk = ensure_rowsweep<K>(s);
    if (rk.rest_probs_f || !rk.n_rest) return;
    std::vector<ScatterProb> pf = rk.rest_host;
    for (auto& pr : pf) {
        pr.load_f = nullptr;
        if (pr.load)
            for (size_t k = 0; k < s.design.loads.size(); ++k)
                if (pr.load == s.op.loads[k]) pr.load_f = s.op_f.loads[k];
    }
    rk.rest_probs_f = s.arena.upload(pf);
}

// `err`: device flag of a timed-out wait of the staged sweep (the LSMR
// loop's ctl->err, or the solver's sweep_err)
template <int K, int MODE, class T>
void launch_rowsweep(within_solver& s, within_solver::RowSweepK& rk, const OpParamsT<T>& op, void* atu, const T* v,
                     T* u, ColState* cur, Ctl* ctl, const int* skip, int store, cudaStream_t st,
                     const T* rhs = nullptr, double* sq_out = nullptr, int sq_stride = 0, int* err = nullptr) {
    RwParams rp = rk.rp;
    rp.atu = atu;
    constexpr int BIN_BYTES = MODE == 2 ? (int)sizeof(T) : 8;
    bool priv;
    const size_t smem = rw_smem_bytes<K, BIN_BYTES>(rp.n_buckets, rp.n_hist, priv);
    rp.hist_private = priv ? 1 : 0;
    bool staged = false;
    if constexpr (K == 1 && (MODE == 0 || MODE == 1) && sizeof(T) == 8) {
        // bulk copies read u from 16-byte aligned chunk starts
        if (rk.ts && ((uintptr_t)u & 15) == 0 && (MODE == 1 || !skip)) {
            TsKernel f = ts_kernel(MODE, rk.ts_nq, rp.n_run, rp.n_hist, op.sqrt_w != nullptr);
            if (f) {
                rp.hist_private = 1;
                int* e = err ? err : (ctl ? &ctl->err : s.sweep_err);
                launch_k(f, rk.grid, RW_THREADS, rk.ts_smem, st, op, rp, rk.ts_slots, v, u, cur, ctl, e);
                staged = true;
            }
        }
    }
    if (!staged) {
        if (rk.simple)
            launch_k(k_rowsweep<K, MODE, T, true>, rk.grid, RW_THREADS, smem, st, op, rp, v, u, cur, ctl, skip, store,
                                                                            rhs, sq_out, sq_stride);
        else
            launch_k(k_rowsweep<K, MODE, T, false>, rk.grid, RW_THREADS, smem, st, op, rp, v, u, cur, ctl, skip, store,
                                                                             rhs, sq_out, sq_stride);
    }
    ++g_launches;
    if (rp.n_fix) {   // the runs crossing range boundaries, after every range has written its partials
        const unsigned fb = (rp.n_fix + 255) / 256;
        if (rk.simple) launch_k(k_rw_fix<K, MODE, T, true>, fb, 256, 0, st, op, rp, ctl, skip);
        else launch_k(k_rw_fix<K, MODE, T, false>, fb, 256, 0, st, op, rp, ctl, skip);
        ++g_launches;
    }
}

// the run combines and full-resolution rest terms of A^T u, raw sums into out
template <int K, class T>
void rowsweep_rest(within_solver& s, within_solver::RowSweepK& rk, const T* u, T* out, const int* skip,
                   cudaStream_t st) {
    if (!rk.n_rest) return;
    if constexpr (sizeof(T) == 8) {
        ScatterF<K, 0> f{rk.rest_probs, u, s.op.sqrt_w, out, nullptr};
        launch_sr<ScatterF<K, 0>, K>(f, rk.rest, 0, rk.rest.n_tiles, skip, st);
    } else {
        ScatterF<K, 0, float> f{rk.rest_probs_f, u, s.op_f.sqrt_w, out, nullptr};
        launch_sr<ScatterF<K, 0, float>, K>(f, rk.rest, 0, rk.rest.n_tiles, skip, st);
    }
}

// WITHIN_SWEEP=0 selects the gather + full segmented-reduction path, any
// other value the row sweep
int env_path(int dflt) {
    if (const char* e = getenv("WITHIN_SWEEP")) return atoi(e) == 0 ? 0 : 2;
    return dflt;
}

// The device vectors of the LSMR loop for K columns (no plans).
within_solver::Work& work_buffers(within_solver& s, int K) {
    auto& w = s.work[kidx(K)];
    if (w.buffers) return w;
    Arena& A = s.arena;
    w.u = A.alloc<double>(s.n_obs * K);
    w.b = A.alloc<double>(s.n_obs * K);
    w.yint = A.alloc<double>(s.n_obs * K);
    w.dm = A.alloc<double>(s.n_obs * K);
    w.v = A.alloc<double>(s.n_dofs * K);
    w.p = A.alloc<double>(s.n_dofs * K);
    w.h = A.alloc<double>(s.n_dofs * K);
    w.hb = A.alloc<double>(s.n_dofs * K);
    w.x = A.alloc<double>(s.n_dofs * K);
    w.partials = A.alloc<double>((size_t)RED_GRID * 3 * 8);
    w.counter = A.alloc<unsigned>(1);
    w.bmax = A.alloc<double>(8);
    w.nonfinite = A.alloc<int>(1);
    w.st = A.alloc<ColState>(2 * 8);
    w.ctl = A.alloc<Ctl>(1);
    w.buffers = true;
    return w;
}

within_solver::Work& ensure_work(within_solver& s, int K) {
    auto& w = s.work[kidx(K)];
    if (w.ready) return w;
    PhaseTrace pt("first use of a column bucket: workspaces and plans");
    work_buffers(s, K);
    if (s.precond && s.precond->kind == 1) schwarz_user_plans(s.schwarz, *s.precond, K);
    ensure_scatter(s, K);
    // Path choice per column count, fixed per process so results stay bitwise
    // reproducible.  WITHIN_SWEEP=0 forces the gather + scatter path.
    const int path = env_path(2);
    s.path[kidx(K)] = path;
    if (path == 2) {
        if (K == 1) ensure_rowsweep<1>(s);
        else if (K == 2) ensure_rowsweep<2>(s);
        else if (K == 4) ensure_rowsweep<4>(s);
        else ensure_rowsweep<8>(s);
    }
    w.ready = true;
    return w;
}

template <int K, int EPI, class T = double>
void scatter(within_solver& s, const T* u, T* out, const ColState* cur, const int* skip, cudaStream_t st) {
    const DevPlan& pl = s.scatter_plan[kidx(K)];
    if constexpr (sizeof(T) == 8) {
        ScatterF<K, EPI> f{s.scatter_probs, u, s.op.sqrt_w, out, cur};
        launch_sr<ScatterF<K, EPI>, K>(f, pl, 0, pl.n_tiles, skip, st);
    } else {
        ScatterF<K, EPI, float> f{s.scatter_probs_f, u, s.op_f.sqrt_w, out, cur};
        launch_sr<ScatterF<K, EPI, float>, K>(f, pl, 0, pl.n_tiles, skip, st);
    }
}

template <int K, class T = double>
void precond_apply(within_solver& s, Ctl* ctl, const T* p, T* v, const int* skip, cudaStream_t st) {
    const uint32_t nd = (uint32_t)s.n_dofs;
    if (!s.precond) {
        launch_k(k_diag_apply<K, T>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, nullptr, p, v, skip ? ctl : nullptr);
        ++g_launches;
    } else if (s.precond->kind == 2) {
        const T* d;
        if constexpr (sizeof(T) == 8) d = s.precond->inv_diag;
        else d = s.precond->inv_diag_f;
        launch_k(k_diag_apply<K, T>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, d, p, v, skip ? ctl : nullptr);
        ++g_launches;
    } else {
        schwarz_apply<K, T>(*s.precond, s.schwarz, p, v, skip, st);
    }
}

// one LSMR iteration at state parity `par`
template <int K>
void iteration(within_solver& s, within_solver::Work& w, int par, cudaStream_t st) {
    ColState* cur = w.st + (size_t)par * 8;
    ColState* nxt = w.st + (size_t)(1 - par) * 8;
    const uint32_t n = (uint32_t)s.n_obs, nd = (uint32_t)s.n_dofs;
    const int* skip = &w.ctl->all_done;
    if (s.path[kidx(K)] == 2) {
        auto& rk = s.rsw[kidx(K)];
        launch_rowsweep<K, 1, double>(s, rk, s.op, rk.atu, w.v, w.u, cur, w.ctl, nullptr, 0, st);
        rowsweep_rest<K, double>(s, rk, w.u, rk.atu, skip, st);
        launch_k(k_ptilde<K>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, rk.atu, w.p, cur, w.ctl);
        ++g_launches;
    } else {
        launch_k(k_gather_update<K>, RED_GRID, RED_THREADS, 0, st, s.op, w.v, w.u, cur, w.ctl, w.partials, w.counter);
        ++g_launches;
        scatter<K, 1>(s, w.u, w.p, cur, skip, st);
    }
    precond_apply<K>(s, w.ctl, w.p, w.v, skip, st);
    for (int j = 0; j < w.ring.cap; ++j) {   // M-MGS against the stored window (bidiag.rs:489-512)
        launch_k(k_reorth_dot<K>, RED_GRID, RED_THREADS, 0, st, nd, j, w.ring, w.v, cur, w.ctl, w.coef, w.partials,
                                                          w.counter);
        launch_k(k_reorth_axpy<K>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, j, w.ring, w.v, w.p, cur, w.ctl, w.coef);
        g_launches += 2;
    }
    launch_k(k_alpha_step<K>, RED_GRID, RED_THREADS, 0, st, nd, w.v, w.p, cur, nxt, w.ctl, w.partials, w.counter);
    ++g_launches;
    launch_k(k_solution_update<K>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, w.v, w.h, w.hb, w.x, nxt, w.ctl, w.ring,
                                                                      w.p);
    ++g_launches;
    (void)n;
}

// The LSMR loop as one graph: a conditional WHILE node whose body is two
// iterations (both state parities) followed by k_loop_cond, which keeps the
// loop going while any column is active.  One launch and one host wait per
// solve, and no iterations run past convergence.  Returns false (and the
// caller replays the two-iteration graph in bursts) if the runtime refuses
// conditional nodes.
template <int K>
bool build_loop_graph(within_solver& s, within_solver::Work& w) {
    if (w.loop_graph) return true;
    if (w.loop_failed) return false;
    PhaseTrace pt("LSMR loop graph capture and instantiation");
    if (const char* e = getenv("WITHIN_GRAPH_LOOP"))
        if (atoi(e) == 0) {
            w.loop_failed = true;
            return false;
        }
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(g);
        w.loop_failed = true;
        return false;
    }
    alignas(cudaGraphNodeParams) unsigned char np_raw[sizeof(cudaGraphNodeParams)] = {};
    cudaGraphNodeParams& np = *reinterpret_cast<cudaGraphNodeParams*>(np_raw);
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, g, nullptr, 0, &np) != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(g);
        w.loop_failed = true;
        return false;
    }
    cudaGraph_t body = np.conditional.phGraph_out[0];
    cudaStream_t cs;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    CK(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    uint64_t before = g_launches;
    iteration<K>(s, w, 0, cs);
    iteration<K>(s, w, 1, cs);
    k_loop_cond<<<1, 1, 0, cs>>>(w.ctl, h);
    w.graph_iters = g_launches - before + 1;
    g_launches = before;
    CK(cudaStreamEndCapture(cs, &body));
    CK(cudaStreamDestroy(cs));
    CK(cudaGraphInstantiate(&w.loop_graph, g, 0));
    CK(cudaGraphDestroy(g));
    return true;
}

template <int K>
void run_lsmr(within_solver& s, within_solver::Work& w, const double* Y, uint32_t k_used, double tol,
              uint64_t maxiter, double* X_out, double* D_out, within_solve_stats* stats, cudaStream_t st,
              double t_setup0, const SolveExt& ext = SolveExt{}, int32_t* stop_out = nullptr) {
    const uint32_t n = (uint32_t)s.n_obs, nd = (uint32_t)s.n_dofs;
    CK(cudaMemsetAsync(w.nonfinite, 0, sizeof(int), st));
    CK(cudaMemsetAsync(w.ctl, 0, sizeof(Ctl), st));
    launch_k(k_load_rhs<K>, RED_GRID, RED_THREADS, 0, st, n, k_used, Y, s.perm, s.op.sqrt_w, w.yint, w.b,
                                                    w.partials, w.counter, w.bmax, w.nonfinite);
    if (ext.x0) {   // warm start: x0 into the interleaved layout (finite check)
        if (!w.x0) w.x0 = s.arena.alloc<double>(s.n_dofs * K);
        launch_k(k_load_x0<K>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, k_used, ext.x0, w.x0, w.nonfinite);
        ++g_launches;
    }
    int nonfinite = 0;
    CK(cudaMemcpyAsync(&nonfinite, w.nonfinite, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (nonfinite)
        throw WError(ERR_INVALID, ext.x0 ? "response and warm start must be finite (a non-finite value was found)"
                                         : "response must be finite (a non-finite value was found)");
    const double t_solve0 = now_s();
    launch_k(k_norm_b<K>, RED_GRID, RED_THREADS, 0, st, n, w.b, w.bmax, w.st, tol, (long long)maxiter, k_used,
                                                  w.ctl, w.partials, w.counter, 0, (int)ext.stale_window,
                                                  ext.stale_threshold);
    if (ext.x0) {   // b <- b - A x0, tolerances kept relative to the original ||b||
        launch_k(k_warm_rhs<K>, RED_GRID, RED_THREADS, 0, st, s.op, w.x0, w.b, w.partials, w.counter, w.bmax);
        launch_k(k_norm_b<K>, RED_GRID, RED_THREADS, 0, st, n, w.b, w.bmax, w.st, tol, (long long)maxiter, k_used,
                                                      w.ctl, w.partials, w.counter, 1, (int)ext.stale_window,
                                                      ext.stale_threshold);
        g_launches += 2;
    }
    launch_k(k_scale_u<K>, grid_for(n, 256, 148 * 16), 256, 0, st, n, w.b, w.u, w.st);
    if (s.path[kidx(K)] == 2) {   // p~ = A^T u through the row sweep (adjoint mode) and its rest
        auto& rk = s.rsw[kidx(K)];
        CK(cudaMemsetAsync(w.p, 0, (size_t)nd * K * sizeof(double), st));   // levels no row reaches stay 0
        launch_rowsweep<K, 0, double>(s, rk, s.op, w.p, nullptr, w.u, nullptr, nullptr, nullptr, 0, st, nullptr,
                                      nullptr, 0, &w.ctl->err);
        rowsweep_rest<K, double>(s, rk, w.u, w.p, nullptr, st);
    } else {
        scatter<K, 0>(s, w.u, w.p, w.st, nullptr, st);
    }
    precond_apply<K>(s, w.ctl, w.p, w.v, nullptr, st);
    launch_k(k_alpha_init<K>, RED_GRID, RED_THREADS, 0, st, nd, w.v, w.p, w.st, w.st + 8, w.ctl, w.partials,
                                                      w.counter);
    launch_k(k_init_vectors<K>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, w.v, w.h, w.hb, w.x, w.st, w.ring, w.p);
    g_launches += 6;
    Ctl ctl{};
    if (build_loop_graph<K>(s, w)) {
        CK(cudaGraphLaunch(w.loop_graph, st));
        CK(cudaMemcpyAsync(&ctl, w.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        g_launches += (uint64_t)ctl.bodies_run * w.graph_iters;
    } else {
    // capture two iterations once per workspace
    if (!w.graph) {
        cudaStream_t cs;
        CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        uint64_t before = g_launches;
        iteration<K>(s, w, 0, cs);
        iteration<K>(s, w, 1, cs);
        w.graph_iters = g_launches - before;
        g_launches = before;
        CK(cudaStreamEndCapture(cs, &g));
        CK(cudaGraphInstantiate(&w.graph, g, 0));
        CK(cudaGraphDestroy(g));
        CK(cudaStreamDestroy(cs));
    }
    uint64_t done_iters = 0;
    uint64_t burst = 2;
    while (true) {
        for (uint64_t b = 0; b < burst; ++b) {
            CK(cudaGraphLaunch(w.graph, st));
            g_launches += w.graph_iters;
        }
        done_iters += 2 * burst;
        CK(cudaMemcpyAsync(&ctl, w.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (ctl.all_done || ctl.err || done_iters >= maxiter + 2) break;
        burst = std::min<uint64_t>(burst * 2, 32);
        uint64_t left = (maxiter + 2 - done_iters + 1) / 2;
        burst = std::max<uint64_t>(1, std::min(burst, left));
    }
    }
    if (ctl.err == 5)
        throw WError(ERR_INDEFINITE, "mlsmr: preconditioner not positive definite (<v, Mv> < 0)");
    if (ctl.err == ERR_WAIT_TIMEOUT)
        throw WError(ERR_CUDA, "row sweep: a bulk copy into shared memory did not complete within 1 s");
    if (ctl.err == ERR_WARM_NONFINITE)
        throw WError(ERR_INVALID, "warm-start residual b - A x0 has a non-finite norm");
    const double t_solve1 = now_s();
    // results
    if (ext.x0) {
        launch_k(k_add_x0<K>, grid_for((uint64_t)nd * K, 256, 148 * 8), 256, 0, st, nd, w.x, w.x0);
        ++g_launches;
    }
    if (K != 1 || !launch_tgather(s, w.x, w.yint, w.dm, true, nullptr, s.sweep_err, st)) {
        launch_k(k_demean<K>, grid_for(n, 256, 148 * 16), 256, 0, st, s.op, w.x, w.yint, w.dm);
        ++g_launches;
    }
    if (D_out) {
        launch_k(k_store_obs<K>, grid_for(n, 256, 148 * 16), 256, 0, st, n, k_used, w.dm, s.perm, D_out);
        ++g_launches;
    }
    if (X_out) {
        launch_k(k_store_dofs<K>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, k_used, w.x, X_out);
        ++g_launches;
    }
    ColState fin[8];
    // the state parity after the loop is whichever buffer was written last:
    // both buffers hold identical done states for finished columns, so read
    // the one with the larger iteration count.
    ColState a[8], b2[8];
    int werr = 0;
    CK(cudaMemcpyAsync(a, w.st, sizeof(ColState) * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(b2, w.st + 8, sizeof(ColState) * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&werr, s.sweep_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (werr) throw WError(ERR_CUDA, "staged gather: a bulk copy into shared memory did not complete within 1 s");
    for (int k = 0; k < 8; ++k) fin[k] = a[k].itn >= b2[k].itn ? a[k] : b2[k];
    if (stop_out)
        for (uint32_t k = 0; k < k_used; ++k) stop_out[k] = fin[k].stop;
    const double t_end = now_s();
    if (stats)
        for (uint32_t k = 0; k < k_used; ++k) {
            const ColState& c = fin[k];
            within_solve_stats& o = stats[k];
            o.converged = (c.stop == STOP_RESID || c.stop == STOP_NORMAL || c.stop == STOP_ZERO_RHS ||
                           c.stop == STOP_INIT_ZERO || c.stop == STOP_WARM_EXACT) ? 1 : 0;
            o.iterations = (uint64_t)c.itn;
            o.residual = (c.stop == STOP_ZERO_RHS || c.stop == STOP_INIT_ZERO || c.stop == STOP_WARM_EXACT)
                             ? 0.0 : fabs(c.zeta_bar) / c.zeta0;
            o.time_setup = t_solve0 - t_setup0;
            o.time_solve = t_solve1 - t_solve0;
            o.time_total = t_end - t_setup0;
        }
}

// ---------------------------------------------------------------------------
// mixed precision (refine.cuh): FP32 copies of the operator's floating data,
// of the preconditioner's factor values and FP32 inner-solve workspaces.
void ensure_mixed_data(within_solver& s) {
    if (s.has_f) return;
    Arena& A = s.arena;
    const HostDesign& D = s.design;
    s.op_f.n = s.op.n;
    s.op_f.Q = s.op.Q;
    for (int t = 0; t < MAXQ; ++t) {
        s.op_f.codes[t] = s.op.codes[t];
        s.op_f.off[t] = s.op.off[t];
        s.op_f.L[t] = s.op.L[t];
        s.op_f.ncol[t] = s.op.ncol[t];
        for (int c = 0; c < MAXC; ++c) s.op_f.load[t][c] = s.op.load[t][c];
    }
    for (size_t k = 0; k < D.loads.size(); ++k) s.op_f.loads[k] = A.upload(cast_vec<float>(D.loads[k]));
    if (s.op.sqrt_w) {
        std::vector<double> sw(s.n_obs);
        CK(cudaMemcpy(sw.data(), s.op.sqrt_w, s.n_obs * sizeof(double), cudaMemcpyDeviceToHost));
        s.op_f.sqrt_w = A.upload(cast_vec<float>(sw));
    }
    std::vector<ScatterProb> pf = s.scatter_host;
    size_t i = 0;
    for (size_t t = 0; t < D.terms.size(); ++t)
        for (size_t c = 0; c < D.terms[t].cols.size(); ++c, ++i)
            pf[i].load_f = D.terms[t].cols[c] < 0 ? nullptr : s.op_f.loads[D.terms[t].cols[c]];
    s.scatter_probs_f = A.upload(pf);
    if (s.precond) ensure_precond_f(*s.precond);
    s.has_f = true;
}

within_solver::MixedWork& ensure_mixed(within_solver& s, int K) {
    auto& m = s.mixed[kidx(K)];
    if (m.ready) return m;
    ensure_work(s, K);   // FP64 rhs staging, reduction scratch, plans
    ensure_mixed_data(s);
    Arena& A = s.arena;
    m.r64 = A.alloc<double>(s.n_obs * K);
    m.g64 = A.alloc<double>(s.n_dofs * K);
    m.x64 = A.alloc<double>(s.n_dofs * K);
    m.t = A.alloc<float>(s.n_obs * K);
    m.res = A.alloc<float>(s.n_dofs * K);
    m.z = A.alloc<float>(s.n_dofs * K);
    m.p = A.alloc<float>(s.n_dofs * K);
    m.q = A.alloc<float>(s.n_dofs * K);
    m.d = A.alloc<float>(s.n_dofs * K);
    m.st = A.alloc<CgCol>(8);
    m.ctl = A.alloc<Ctl>(1);
    if (s.precond && s.precond->kind == 1) schwarz_user_work_f(s.schwarz, *s.precond, K);
    if (s.path[kidx(K)] == 2) {
        if (K == 1) ensure_rowsweep_f<1>(s);
        else if (K == 2) ensure_rowsweep_f<2>(s);
        else if (K == 4) ensure_rowsweep_f<4>(s);
        else ensure_rowsweep_f<8>(s);
    }
    m.ready = true;
    return m;
}

// one inner CG iteration in FP32 storage
template <int K>
void cg_iteration(within_solver& s, within_solver::Work& w, within_solver::MixedWork& m, cudaStream_t st) {
    const uint32_t nd = (uint32_t)s.n_dofs;
    const int* skip = &m.ctl->all_done;
    if (s.path[kidx(K)] == 2) {
        auto& rk = s.rsw[kidx(K)];
        launch_rowsweep<K, 2, float>(s, rk, s.op_f, m.q, m.p, m.t, nullptr, m.ctl, skip, rk.rest_needs_rows ? 1 : 0,
                                     st);
        rowsweep_rest<K, float>(s, rk, m.t, m.q, skip, st);
    } else {
        launch_k(k_apply<K, float>, grid_for(s.n_obs, 256 * 4, 148 * 8), 256, 0, st, s.op_f, m.p, m.t, skip);
        ++g_launches;
        scatter<K, 0, float>(s, m.t, m.q, nullptr, skip, st);
    }
    launch_k(k_cg_alpha<K, float>, RED_GRID, RED_THREADS, 0, st, nd, m.p, m.q, m.st, m.ctl, w.partials, w.counter);
    launch_k(k_cg_update<K, float>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, m.p, m.q, m.d, m.res, m.st, m.ctl);
    g_launches += 2;
    precond_apply<K, float>(s, m.ctl, m.res, m.z, skip, st);
    launch_k(k_cg_beta<K, float>, RED_GRID, RED_THREADS, 0, st, nd, m.res, m.z, m.st, m.ctl, w.partials, w.counter);
    launch_k(k_cg_dir<K, float>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, m.z, m.p, m.st, m.ctl);
    g_launches += 2;
}

template <int K>
void build_cg_loop(within_solver& s, within_solver::Work& w, within_solver::MixedWork& m) {
    if (m.loop_graph) return;
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    alignas(cudaGraphNodeParams) unsigned char np_raw[sizeof(cudaGraphNodeParams)] = {};
    cudaGraphNodeParams& np = *reinterpret_cast<cudaGraphNodeParams*>(np_raw);
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, nullptr, 0, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    cudaStream_t cs;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    CK(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = g_launches;
    cg_iteration<K>(s, w, m, cs);
    k_loop_cond<<<1, 1, 0, cs>>>(m.ctl, h);
    m.body_launches = g_launches - before + 1;
    g_launches = before;
    CK(cudaStreamEndCapture(cs, &body));
    CK(cudaStreamDestroy(cs));
    CK(cudaGraphInstantiate(&m.loop_graph, g, 0));
    CK(cudaGraphDestroy(g));
}

// One refinement step's set-up: r = b - A x, ||r||, g = A^T r in FP64, the
// FP32 copy of g, z = M^-1 g, rho0 and the outer stopping tests (k_cg_init).
template <int K>
void mixed_pre(within_solver& s, within_solver::Work& w, within_solver::MixedWork& m, cudaStream_t st, int first,
               int use_h, cudaGraphConditionalHandle h_in) {
    const uint32_t nd = (uint32_t)s.n_dofs;
    if (s.path[kidx(K)] == 2) {   // r = b - A x, ||r||^2 and g = A^T r in one row sweep
        auto& rk = s.rsw[kidx(K)];
        launch_rowsweep<K, 3, double>(s, rk, s.op, m.g64, m.x64, m.r64, nullptr, nullptr, nullptr,
                                      rk.rest_needs_rows ? 1 : 0, st, w.b, &m.st[0].rnorm2,
                                      (int)(sizeof(CgCol) / sizeof(double)));
        rowsweep_rest<K, double>(s, rk, m.r64, m.g64, nullptr, st);
    } else {
        launch_k(k_resid64<K>, RED_GRID, RED_THREADS, 0, st, s.op, m.x64, w.b, m.r64, m.st, w.partials, w.counter);
        ++g_launches;
        scatter<K, 0>(s, m.r64, m.g64, nullptr, nullptr, st);
    }
    launch_k(k_cg_start<K, float>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, m.g64, m.res, m.d);
    precond_apply<K, float>(s, m.ctl, m.res, m.z, nullptr, st);
    launch_k(k_cg_init<K, float>, RED_GRID, RED_THREADS, 0, st, nd, m.res, m.z, m.p, m.st, m.ctl, first, w.partials,
                                                           w.counter, use_h, h_in);
    g_launches += 2;
}

// The whole mixed solve as one graph: a WHILE node over refinement steps
// whose body is [mixed_pre, a WHILE node over CG iterations, x += d,
// k_outer_cond].  One launch and one host wait per solve; returns false if
// the runtime refuses nested conditional nodes (the host then drives the
// refinement steps).
template <int K>
bool build_mixed_graph(within_solver& s, within_solver::Work& w, within_solver::MixedWork& m) {
    if (m.solve_graph) return true;
    if (m.solve_graph_failed) return false;
    const uint32_t nd = (uint32_t)s.n_dofs;
    auto cond_params = [](cudaGraphConditionalHandle h, unsigned char* raw) -> cudaGraphNodeParams& {
        cudaGraphNodeParams& np = *reinterpret_cast<cudaGraphNodeParams*>(raw);
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        return np;
    };
    cudaGraph_t g = nullptr;
    cudaStream_t cs = nullptr;
    bool ok = false;
    do {
        if (cudaGraphCreate(&g, 0) != cudaSuccess) break;
        cudaGraphConditionalHandle h_out, h_in;
        if (cudaGraphConditionalHandleCreate(&h_out, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) break;
        alignas(cudaGraphNodeParams) unsigned char raw_out[sizeof(cudaGraphNodeParams)] = {};
        cudaGraphNodeParams& np_out = cond_params(h_out, raw_out);
        cudaGraphNode_t n_out;
        if (cudaGraphAddNode(&n_out, g, nullptr, 0, &np_out) != cudaSuccess) break;
        cudaGraph_t body = np_out.conditional.phGraph_out[0];
        if (cudaGraphConditionalHandleCreate(&h_in, body, 0, 0) != cudaSuccess) break;
        if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) break;
        const uint64_t l0 = g_launches;
        CK(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        mixed_pre<K>(s, w, m, cs, -1, 1, h_in);
        cudaStreamCaptureStatus cst;
        cudaGraph_t capg;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        CK(cudaStreamGetCaptureInfo(cs, &cst, nullptr, &capg, &deps, &ndeps));
        alignas(cudaGraphNodeParams) unsigned char raw_in[sizeof(cudaGraphNodeParams)] = {};
        cudaGraphNodeParams& np_in = cond_params(h_in, raw_in);
        cudaGraphNode_t n_in;
        CK(cudaGraphAddNode(&n_in, capg, deps, ndeps, &np_in));
        cudaGraph_t inner = np_in.conditional.phGraph_out[0];
        CK(cudaStreamUpdateCaptureDependencies(cs, &n_in, 1, cudaStreamSetCaptureDependencies));
        m.pre_launches = g_launches - l0;
        const uint64_t l1 = g_launches;
        launch_k(k_add_delta<K, float>, grid_for(nd, 256, 148 * 8), 256, 0, cs, nd, m.d, m.x64);
        k_outer_cond<<<1, 1, 0, cs>>>(m.st, m.ctl, h_out);
        m.post_launches = g_launches - l1 + 2;
        CK(cudaStreamEndCapture(cs, &body));
        const uint64_t l2 = g_launches;
        CK(cudaStreamBeginCaptureToGraph(cs, inner, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        cg_iteration<K>(s, w, m, cs);
        k_loop_cond<<<1, 1, 0, cs>>>(m.ctl, h_in);
        m.body_launches = g_launches - l2 + 1;
        CK(cudaStreamEndCapture(cs, &inner));
        g_launches = l0;
        CK(cudaGraphInstantiate(&m.solve_graph, g, 0));
        ok = true;
    } while (false);
    if (cs) cudaStreamDestroy(cs);
    if (g) cudaGraphDestroy(g);
    if (!ok) {
        cudaGetLastError();
        m.solve_graph_failed = true;
    }
    return ok;
}

// Mixed-precision solve of K columns: FP64 refinement steps around FP32-storage
// CG on the normal equations (refine.cuh); same outputs as run_lsmr.
template <int K>
void run_mixed(within_solver& s, const double* Y, uint32_t k_used, double tol, uint64_t maxiter, double* X_out,
               double* D_out, within_solve_stats* stats, cudaStream_t st, double t_setup0) {
    auto& w = ensure_work(s, K);
    auto& m = ensure_mixed(s, K);
    const uint32_t n = (uint32_t)s.n_obs, nd = (uint32_t)s.n_dofs;
    CK(cudaMemsetAsync(w.nonfinite, 0, sizeof(int), st));
    launch_k(k_load_rhs<K>, RED_GRID, RED_THREADS, 0, st, n, k_used, Y, s.perm, s.op.sqrt_w, w.yint, w.b, w.partials,
                                                    w.counter, w.bmax, w.nonfinite);
    ++g_launches;
    int nonfinite = 0;
    CK(cudaMemcpyAsync(&nonfinite, w.nonfinite, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (nonfinite) throw WError(ERR_INVALID, "response must be finite (a non-finite value was found)");
    const double t_solve0 = now_s();
    build_cg_loop<K>(s, w, m);
    CK(cudaMemsetAsync(m.x64, 0, (size_t)nd * K * sizeof(double), st));
    double floor = CG_FLOOR;
    if (const char* e = getenv("WITHIN_CG_FLOOR")) floor = atof(e);
    k_cg_setup<<<1, 1, 0, st>>>(m.st, (int)k_used, tol, (long long)std::min<uint64_t>(maxiter, (uint64_t)1 << 40),
                                m.ctl, floor);
    ++g_launches;
    CgCol fin[8];
    Ctl ctl{};
    const char* gl = getenv("WITHIN_GRAPH_LOOP");
    const bool device_driven = !(gl && atoi(gl) == 0) && build_mixed_graph<K>(s, w, m);
    if (device_driven) {
        CK(cudaGraphLaunch(m.solve_graph, st));
        CK(cudaMemcpyAsync(&ctl, m.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        g_launches += (uint64_t)ctl.outer * (m.pre_launches + m.post_launches) +
                      (uint64_t)ctl.bodies_run * m.body_launches;
    }
    for (int outer = 0; !device_driven; ++outer) {
        mixed_pre<K>(s, w, m, st, outer == 0 ? 1 : 0, 0, cudaGraphConditionalHandle{});
        CK(cudaMemcpyAsync(&ctl, m.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (ctl.all_done || ctl.err) break;
        const int runs0 = ctl.bodies_run;
        if (const char* e = getenv("WITHIN_GRAPH_LOOP"); e && atoi(e) == 0) {
            // plain launches, one host check per iteration (for profilers that
            // do not follow conditional graph bodies)
            for (uint64_t it = 0; it <= maxiter; ++it) {
                cg_iteration<K>(s, w, m, st);
                CK(cudaMemcpyAsync(&ctl, m.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                if (ctl.all_done || ctl.err) break;
            }
            ctl.bodies_run = runs0;
        } else {
            CK(cudaGraphLaunch(m.loop_graph, st));
        }
        launch_k(k_add_delta<K, float>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, m.d, m.x64);
        ++g_launches;
        CK(cudaMemcpyAsync(&ctl, m.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        g_launches += (uint64_t)(ctl.bodies_run - runs0) * m.body_launches;
        if (ctl.err || outer > 64) break;
    }
    CK(cudaMemcpyAsync(fin, m.st, sizeof(CgCol) * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (ctl.err == 5)
        throw WError(ERR_INDEFINITE, "mixed solve: preconditioner not positive definite (<g, M g> < 0)");
    const double t_solve1 = now_s();
    if (K != 1 || !launch_tgather(s, m.x64, w.yint, w.dm, true, nullptr, s.sweep_err, st)) {
        launch_k(k_demean<K>, grid_for(n, 256, 148 * 16), 256, 0, st, s.op, m.x64, w.yint, w.dm);
        ++g_launches;
    }
    if (D_out) {
        launch_k(k_store_obs<K>, grid_for(n, 256, 148 * 16), 256, 0, st, n, k_used, w.dm, s.perm, D_out);
        ++g_launches;
    }
    if (X_out) {
        launch_k(k_store_dofs<K>, grid_for(nd, 256, 148 * 8), 256, 0, st, nd, k_used, m.x64, X_out);
        ++g_launches;
    }
    int werr = 0;
    CK(cudaMemcpyAsync(&werr, s.sweep_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (werr) throw WError(ERR_CUDA, "staged gather: a bulk copy into shared memory did not complete within 1 s");
    const double t_end = now_s();
    if (stats)
        for (uint32_t k = 0; k < k_used; ++k) {
            const CgCol& c = fin[k];
            within_solve_stats& o = stats[k];
            o.converged = (c.stop == STOP_RESID || c.stop == STOP_NORMAL || c.stop == STOP_ZERO_RHS ||
                           c.stop == STOP_INIT_ZERO) ? 1 : 0;
            o.iterations = (uint64_t)c.itn;
            o.residual = c.bnorm > 0.0 ? sqrt(c.rnorm2) / c.bnorm : 0.0;
            o.time_setup = t_solve0 - t_setup0;
            o.time_solve = t_solve1 - t_solve0;
            o.time_total = t_end - t_setup0;
        }
}

// The reorthogonalisation window of a workspace: cap = min(local_size, m, n)
// pairs (bidiag.rs:113-217).  The graphs bake the window in, so a change of
// local_size rebuilds them.
void set_ring(within_solver& s, within_solver::Work& w, int K, uint64_t local_size) {
    const uint64_t cap = std::min<uint64_t>(local_size, std::min<uint64_t>(s.n_obs, s.n_dofs));
    if ((int)cap == w.ring.cap) return;
    if (cap > 4096) throw WError(ERR_UNSUPPORTED, "local_size above 4096 is not supported");
    if (w.graph) cudaGraphExecDestroy(w.graph);
    if (w.loop_graph) cudaGraphExecDestroy(w.loop_graph);
    w.graph = nullptr;
    w.loop_graph = nullptr;
    if (cap > w.ring_alloc) {
        w.ring.V = s.arena.alloc<double>(cap * s.n_dofs * K);
        w.ring.P = s.arena.alloc<double>(cap * s.n_dofs * K);
        w.ring_alloc = cap;
    }
    if (!w.coef) w.coef = s.arena.alloc<double>(8);
    w.ring.cap = (int)cap;
}

void dispatch_solve(within_solver& s, const double* Y_dev, uint64_t k, double tol, uint64_t maxiter,
                    double* X_dev, double* D_dev, within_solve_stats* stats, cudaStream_t st,
                    uint64_t local_size = 0, const SolveExt& ext = SolveExt{}, int32_t* stop_out = nullptr) {
    const double t0 = now_s();
    if (local_size && s.precision == WITHIN_PRECISION_MIXED)
        throw WError(ERR_UNSUPPORTED, "local_size (windowed reorthogonalisation) applies to the FP64 LSMR solve; "
                                      "the mixed-precision solve refines instead");
    if ((ext.x0 || ext.stale_window) && s.precision == WITHIN_PRECISION_MIXED)
        throw WError(ERR_UNSUPPORTED, "warm starts and escalation apply to the FP64 LSMR solve");
    for (uint64_t c0 = 0; c0 < k; c0 += 8) {
        const uint32_t kk = (uint32_t)std::min<uint64_t>(8, k - c0);
        const int K = k_bucket(kk);
        auto& w = ensure_work(s, K);
        if (s.precision != WITHIN_PRECISION_MIXED) set_ring(s, w, K, local_size);
        const double* Y = Y_dev + c0 * s.n_obs;
        double* X = X_dev ? X_dev + c0 * s.n_dofs : nullptr;
        double* D = D_dev ? D_dev + c0 * s.n_obs : nullptr;
        within_solve_stats* S = stats ? stats + c0 : nullptr;
        SolveExt e = ext;
        if (e.x0) e.x0 += c0 * s.n_dofs;
        int32_t* so = stop_out ? stop_out + c0 : nullptr;
        if (s.precision == WITHIN_PRECISION_MIXED) {
            switch (K) {
                case 1: run_mixed<1>(s, Y, kk, tol, maxiter, X, D, S, st, t0); break;
                case 2: run_mixed<2>(s, Y, kk, tol, maxiter, X, D, S, st, t0); break;
                case 4: run_mixed<4>(s, Y, kk, tol, maxiter, X, D, S, st, t0); break;
                default: run_mixed<8>(s, Y, kk, tol, maxiter, X, D, S, st, t0); break;
            }
            continue;
        }
        switch (K) {
            case 1: run_lsmr<1>(s, w, Y, kk, tol, maxiter, X, D, S, st, t0, e, so); break;
            case 2: run_lsmr<2>(s, w, Y, kk, tol, maxiter, X, D, S, st, t0, e, so); break;
            case 4: run_lsmr<4>(s, w, Y, kk, tol, maxiter, X, D, S, st, t0, e, so); break;
            default: run_lsmr<8>(s, w, Y, kk, tol, maxiter, X, D, S, st, t0, e, so); break;
        }
    }
}

void validate_opts(const within_lsmr_options* o, double& tol, uint64_t& maxiter, uint64_t& local_size) {
    tol = 1e-8;
    maxiter = 1000;
    local_size = 0;
    if (o) {
        tol = o->tol;
        maxiter = o->maxiter;
        local_size = o->local_size;
    }
    if (!std::isfinite(tol) || tol < 0.0)
        throw WError(ERR_INVALID, "tolerance must be finite and nonnegative, got " + std::to_string(tol));

}

template <class F>
int guarded(F f) {
    try {
        f();
        return WITHIN_OK;
    } catch (const WError& e) {
        g_err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_err = "host allocation failed";
        return WITHIN_ERR_CUDA;
    } catch (const std::exception& e) {
        g_err = e.what();
        return WITHIN_ERR_CUDA;
    }
}

// prepare_single: also make the single-column workspaces and Schwarz plans
// (the first solve's set-up), overlapping the preconditioner's host build and
// upload; solver sets, which solve column batches, leave them to first use.
within_solver* make_solver(const within_design* d, const double* weights, const within_precond_config* cfg,
                           const within_preconditioner* prebuilt, int device, const within_tuning* tuning = nullptr,
                           bool prepare_single = true) {
    if (!d) throw WError(ERR_INVALID, "design is NULL");
    if (device < 0) CK(cudaGetDevice(&device));
    set_device(device);
    auto s = std::make_unique<within_solver>();
    s->device = device;
    CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->sweep_err = s->arena.alloc<int>(1);
    s->schwarz.tuning = resolve_tuning(tuning);
    pdl_setup(device);
    std::vector<EffectIn> effs;
    for (size_t e = 0; e < d->levels.size(); ++e) {
        EffectIn ef;
        ef.levels = d->levels[e].data();
        ef.intercept = d->intercept[e] != 0;
        for (size_t j : d->slope_of[e]) ef.slopes.push_back(d->slopes[j].data());
        effs.push_back(ef);
    }
    PhaseTrace pt_all("Solver::new total");
    {
        PhaseTrace pt("design build (locality sort)");
        s->design = make_design(d->n_obs, effs);
    }
    HostDesign& D = s->design;
    s->n_obs = D.n_obs;
    s->n_dofs = D.n_dofs;
    // Design::validate_weights (domain.rs:261-279), then permute in
    std::vector<double> w;
    if (weights) {
        for (uint64_t i = 0; i < D.n_obs; ++i)
            if (!(weights[i] >= 0.0 && std::isfinite(weights[i])))
                throw WError(ERR_BUILD, "weight at index " + std::to_string(i) +
                                            " must be finite and non-negative, got " + std::to_string(weights[i]));
        w.resize(D.n_obs);
        for (uint64_t i = 0; i < D.n_obs; ++i) w[i] = D.obs_perm.empty() ? weights[i] : weights[D.obs_perm[i]];
    }
    s->reparam = build_reparam(D, weights ? w.data() : nullptr);
    // codes and loads of the design operator on the device (the GPU cross-tabs
    // of the preconditioner's set-up read them)
    Arena& A = s->arena;
    OpParams& op = s->op;
    {
        PhaseTrace pt("design codes upload");
        op.n = (uint32_t)D.n_obs;
        op.Q = (int)D.terms.size();
        for (size_t k = 0; k < D.loads.size(); ++k) op.loads[k] = A.upload(D.loads[k]);
        for (int t = 0; t < op.Q; ++t) {
            const Term& T = D.terms[t];
            op.codes[t] = A.upload(D.codes[t]);
            op.off[t] = T.offset;
            op.L[t] = T.n_levels;
            op.ncol[t] = (int)T.cols.size();
            for (size_t c = 0; c < T.cols.size(); ++c) op.load[t][c] = T.cols[c];
        }
    }
    // preconditioner (operator/schwarz.rs:231-270)
    BuildResult pre;
    PrecondCfg pre_cfg;
    std::vector<CrossTab> pre_xtabs;
    std::exception_ptr pre_err;
    std::thread pre_thread;
    // the GPU cross-tabs: one host thread and stream per pair, each pair's
    // future ready once its cross-tab is back on the host
    std::unique_ptr<Arena> xt_arena;
    std::vector<std::thread> xt_threads;
    std::vector<std::promise<void>> xt_done;
    std::vector<std::shared_future<void>> xt_ready;
    struct Joiner {   // the host build and the cross-tab threads never outlive this frame, whatever throws
        std::thread& t;
        std::vector<std::thread>& xt;
        ~Joiner() {
            for (auto& x : xt)
                if (x.joinable()) x.join();
            if (t.joinable()) t.join();
        }
    } pre_join{pre_thread, xt_threads};
    if (prebuilt) {
        if (prebuilt->n != D.n_dofs)
            throw WError(ERR_DIMENSION, "prebuilt preconditioner shape (" + std::to_string(prebuilt->n) + "x" +
                                            std::to_string(prebuilt->n) + ") does not match design DOF count " +
                                            std::to_string(D.n_dofs));
        if (prebuilt->device != device) throw WError(ERR_INVALID, "prebuilt preconditioner lives on another device");
        s->precond = const_cast<within_preconditioner*>(prebuilt);
        ++s->precond->refs;
    } else {
        PrecondCfg pc;
        if (cfg) {
            pc.kind = cfg->kind;
            pc.ac_seed = cfg->approx_chol_seed;
            pc.ac_split = cfg->approx_chol_split;
            pc.schur_exact = cfg->schur_exact != 0;
            pc.schur_seed = cfg->schur_seed;
            pc.schur_split = std::max<uint32_t>(1, cfg->schur_split);
            pc.dense_threshold = cfg->dense_threshold;
            pc.scaling_tol = cfg->scaling_tolerance;
            pc.scaling_max_sweeps = cfg->scaling_max_sweeps;
            pc.scaling_error = cfg->scaling_error != 0;
            if (pc.kind < 0 || pc.kind > 2) throw WError(ERR_INVALID, "unknown preconditioner kind");
        }
        // stop rules of the round-parallel factor (see PrecondCfg): the
        // caller's tuning record, else the environment overrides
        if (tuning) {
            pc.core_dense_max = tuning->core_dense_max;
            pc.core_min_frac = tuning->core_min_frac;
            pc.max_rounds = tuning->max_rounds;
            pc.core_small = tuning->core_small;
            pc.core_dense_late = tuning->core_dense_late;
        } else {
            if (const char* e = getenv("WITHIN_CORE_DENSE_MAX")) pc.core_dense_max = (uint32_t)atol(e);
            if (const char* e = getenv("WITHIN_CORE_MIN_FRAC")) pc.core_min_frac = atof(e);
            if (const char* e = getenv("WITHIN_MAX_ROUNDS")) pc.max_rounds = (uint32_t)atol(e);
            if (const char* e = getenv("WITHIN_CORE_SMALL")) pc.core_small = (uint32_t)atol(e);
            if (const char* e = getenv("WITHIN_CORE_DENSE_LATE")) pc.core_dense_late = (uint32_t)atol(e);
        }
        // the host build runs on its own thread while this one uploads the
        // design and builds its scatter orders and sweep plans (both only read
        // the host design)
        pre_cfg = pc;
        // the cross-tabs of the additive-Schwarz set-up on the GPU
        const int gx = s->schwarz.tuning.gpu_cross_tab;
        const bool use_xtab = pc.kind == 1 && (gx >= 2 || (gx == 1 && D.n_obs >= XTAB_MIN_OBS));
        if (use_xtab) {
            double* w_dev = nullptr;
            xt_arena.reset(new Arena());
            if (weights) w_dev = xt_arena->upload(w);
            const std::vector<ChannelPair> cps = schwarz_channel_pairs(D);
            pre_xtabs.resize(cps.size());
            xt_done.resize(cps.size());
            for (auto& p : xt_done) xt_ready.push_back(p.get_future().share());
            // the pairs' device work and their copies back (page faults of
            // fresh host memory included) overlap, and the host build starts
            // each pair as soon as its cross-tab is back
            for (size_t i = 0; i < cps.size(); ++i)
                xt_threads.emplace_back([&, i, cp = cps[i], w_dev] {
                    cudaStream_t st = nullptr;
                    try {
                        set_device(device);
                        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
                        gpu_cross_tab(D.n_obs, op.codes[cp.term_a], D.terms[cp.term_a].n_levels,
                                      op.codes[cp.term_b], D.terms[cp.term_b].n_levels, w_dev,
                                      cp.load_a < 0 ? nullptr : op.loads[cp.load_a],
                                      cp.load_b < 0 ? nullptr : op.loads[cp.load_b], pre_xtabs[i], st);
                        xt_done[i].set_value();
                    } catch (const std::exception& e) {
                        xt_done[i].set_exception(std::make_exception_ptr(WError(ERR_CUDA, e.what())));
                    } catch (...) {
                        xt_done[i].set_exception(std::current_exception());
                    }
                    if (st) cudaStreamDestroy(st);
                });
        }
        pre_thread = std::thread([&, use_xtab] {
            try {
                PhaseTrace pt("preconditioner host build");
                pre = build_preconditioner(D, weights ? w.data() : nullptr, pre_cfg, use_xtab ? &pre_xtabs : nullptr,
                                           use_xtab ? &xt_ready : nullptr);
            } catch (...) {
                pre_err = std::current_exception();
            }
        });
    }
    // the rest of the design operator on the device
    PhaseTrace pt_op("design upload and scatter orders");
    if (weights) {
        std::vector<double> sw(w);
        for (double& x : sw) x = std::sqrt(x);
        op.sqrt_w = A.upload(sw);
    }
    if (!D.obs_perm.empty()) s->perm = A.upload(D.obs_perm);
    // scatter problems: level-sorted order per term (identity when sorted)
    s->level_ptr_host.resize(op.Q);
    for (int t = 0; t < op.Q; ++t) {
        const Term& T = D.terms[t];
        const auto& codes = D.codes[t];
        std::vector<uint32_t>& lp = s->level_ptr_host[t];
        level_counts(codes.data(), D.n_obs, T.n_levels, lp);
        uint32_t* dlp = A.upload(lp);
        uint32_t* order = nullptr;
        if (!T.sorted) {
            std::vector<uint32_t> perm(D.n_obs);
            stable_argsort_u32(codes.data(), D.n_obs, T.n_levels, perm.data());
            order = A.upload(perm);
        }
        for (size_t c = 0; c < T.cols.size(); ++c) {
            ScatterProb sp{};
            sp.seg_ptr = dlp;
            sp.order = order;
            sp.load = T.cols[c] < 0 ? nullptr : op.loads[T.cols[c]];
            sp.out_off = (uint32_t)(T.offset + c * T.n_levels);
            s->scatter_host.push_back(sp);
        }
    }
    s->scatter_probs = A.upload(s->scatter_host);
    {   // single-column plans of the sweep need only the design: built at construction
        // (while the preconditioner's host build, if any, runs on its thread)
        PhaseTrace pt("single-column sweep plans");
        ensure_scatter(*s, 1);
        if (env_path(2) == 2) ensure_rowsweep<1>(*s);
    }
    pt_op.done();
    if (prepare_single) {
        PhaseTrace pt("single-column workspaces");
        work_buffers(*s, 1);
    }
    for (auto& x : xt_threads) x.join();
    xt_threads.clear();
    xt_arena.reset();
    if (pre_thread.joinable()) {
        PhaseTrace pt_wait("wait for the preconditioner host build");
        pre_thread.join();
        pt_wait.done();
        if (pre_err) std::rethrow_exception(pre_err);
        PhaseTrace pt_up("preconditioner upload");
        s->n_warnings = pre.n_warnings;
        if (pre.kind != 0) {
            auto* P = new within_preconditioner();
            P->device = device;
            P->kind = pre.kind;
            P->n = (uint32_t)D.n_dofs;
            try {
                if (pre.kind == 2) {
                    P->inv_diag = P->arena.upload(pre.inv_diag);
                    P->host_inv_diag = pre.inv_diag;
                } else {
                    // the single-column plans read only the host image: built
                    // on a second thread while the image uploads
                    P->host = std::move(pre.schwarz);
                    std::exception_ptr plan_err;
                    std::thread plans;
                    if (prepare_single)
                        plans = std::thread([&] {
                            try {
                                set_device(device);
                                schwarz_user_plans(s->schwarz, *P, 1);
                            } catch (...) {
                                plan_err = std::current_exception();
                            }
                        });
                    try {
                        upload_schwarz_image(*P);
                    } catch (...) {
                        if (plans.joinable()) plans.join();
                        throw;
                    }
                    if (plans.joinable()) plans.join();
                    if (plan_err) std::rethrow_exception(plan_err);
                }
            } catch (...) {
                delete P;
                throw;
            }
            s->precond = P;
        }
    }
    CK(cudaDeviceSynchronize());
    return s.release();
}

// Large host copies (the staging of the host entry points) split over host
// threads: one thread moves ~5-10 GB/s, and first touches of freshly
// allocated caller buffers fault page by page, so a single-threaded copy of a
// 10M-row column costs more than the device solve.
void par_memcpy(void* dst, const void* src, size_t bytes) {
    const size_t piece = (size_t)1 << 20;   // pieces of 1 MiB on the host pool
    const size_t n = (bytes + piece - 1) / piece;
    if (n <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    par_for_each(n, [&](size_t j) {
        const size_t a = j * piece, len = std::min(piece, bytes - a);
        std::memcpy((char*)dst + a, (const char*)src + a, len);
    });
}

// Whether a host pointer is page-locked memory the DMA engines can read or
// write directly (cudaHostAlloc / cudaHostRegister, torch pin_memory).
bool is_pinned(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Host <-> device copies of the host entry points.  A page-locked caller
// buffer is copied directly by one cudaMemcpyAsync; a pageable one goes
// through the solver's two pinned staging slots in chunks, the host copy of
// one chunk (on host threads) overlapping the DMA of the other.
struct Staging {
    within_solver& s;
    cudaStream_t st;
    static constexpr size_t CHUNK = (size_t)16 << 20;   // bytes per slot
    // copies up to this size skip the slots (allocating them costs more than
    // the overlap gains)
    static constexpr size_t SMALL = (size_t)32 << 20;
    char* slot[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    Staging(within_solver& s_, cudaStream_t st_) : s(s_), st(st_) {}
    ~Staging() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
    void ensure() {
        if (!s.pin) {
            CK(cudaMallocHost(&s.pin, 2 * CHUNK));
            s.pin_n = 2 * CHUNK / sizeof(double);
        }
        slot[0] = (char*)s.pin;
        slot[1] = (char*)s.pin + CHUNK;
        for (auto& e : ev)
            if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    void h2d(void* dst, const void* src, size_t bytes) {
        if (!bytes) return;
        if (is_pinned(src) || bytes <= SMALL) {   // small pageable copies: the driver's own staging
            CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
            return;
        }
        ensure();
        for (size_t off = 0, i = 0; off < bytes; off += CHUNK, ++i) {
            const int j = (int)(i & 1);
            const size_t len = std::min(CHUNK, bytes - off);
            if (i >= 2) CK(cudaEventSynchronize(ev[j]));   // the slot's previous DMA has read it
            par_memcpy(slot[j], (const char*)src + off, len);
            CK(cudaMemcpyAsync((char*)dst + off, slot[j], len, cudaMemcpyHostToDevice, st));
            CK(cudaEventRecord(ev[j], st));
        }
    }
    // device -> host; returns after the data is in dst
    void d2h(void* dst, const void* src, size_t bytes) {
        if (!bytes) return;
        if (is_pinned(dst) || bytes <= SMALL) {
            CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            return;
        }
        ensure();
        const size_t n_chunks = (bytes + CHUNK - 1) / CHUNK;
        auto issue = [&](size_t i) {
            const int j = (int)(i & 1);
            const size_t off = i * CHUNK, len = std::min(CHUNK, bytes - off);
            CK(cudaMemcpyAsync(slot[j], (const char*)src + off, len, cudaMemcpyDeviceToHost, st));
            CK(cudaEventRecord(ev[j], st));
        };
        issue(0);
        if (n_chunks > 1) issue(1);
        for (size_t i = 0; i < n_chunks; ++i) {
            const int j = (int)(i & 1);
            const size_t off = i * CHUNK, len = std::min(CHUNK, bytes - off);
            CK(cudaEventSynchronize(ev[j]));
            par_memcpy((char*)dst + off, slot[j], len);
            if (i + 2 < n_chunks) issue(i + 2);   // the slot is free again
        }
    }
};

void host_solve(within_solver& s, const double* Y, uint64_t k, const within_lsmr_options* opts, double* X,
                double* Dm, within_solve_stats* stats) {
    double tol;
    uint64_t maxiter, ls;
    validate_opts(opts, tol, maxiter, ls);
    std::lock_guard<std::mutex> g(s.mu);
    set_device(s.device);
    const uint64_t n = s.n_obs, nd = s.n_dofs;
    double* dY = nullptr;
    double* dX = nullptr;
    double* dD = nullptr;
    CK(cudaMallocAsync(&dY, k * n * sizeof(double), s.stream));
    CK(cudaMallocAsync(&dX, k * nd * sizeof(double), s.stream));
    CK(cudaMallocAsync(&dD, k * n * sizeof(double), s.stream));
    struct Free {
        cudaStream_t st;
        double *a, *b, *c;
        ~Free() {
            cudaFreeAsync(a, st);
            cudaFreeAsync(b, st);
            cudaFreeAsync(c, st);
        }
    } fr{s.stream, dY, dX, dD};
    Staging io(s, s.stream);
    {
        PhaseTrace pt("host -> device copy of the right-hand sides");
        io.h2d(dY, Y, k * n * sizeof(double));
    }
    dispatch_solve(s, dY, k, tol, maxiter, X ? dX : nullptr, Dm ? dD : nullptr, stats, s.stream, ls);
    PhaseTrace pt_out("device -> host copy of the results");
    if (Dm) io.d2h(Dm, dD, k * n * sizeof(double));
    if (X) {
        io.d2h(X, dX, k * nd * sizeof(double));
        if (s.reparam.active())
            for (uint64_t j = 0; j < k; ++j) s.reparam.back_transform(X + j * nd);
    }
}

// Runs fn(i) for i in [0, n) on `threads` host threads (device `dev` current
// in each); the first failure (code, message) is rethrown on the caller.
template <class F>
void parallel_for(uint64_t n, uint32_t threads, int dev, F fn) {
    std::atomic<uint64_t> next{0};
    std::mutex emu;
    int ecode = 0;
    std::string emsg;
    auto work = [&] {
        try {
            set_device(dev);
            for (uint64_t i; (i = next.fetch_add(1)) < n;) {
                {
                    std::lock_guard<std::mutex> g(emu);
                    if (ecode) return;
                }
                fn(i);
            }
        } catch (const WError& e) {
            std::lock_guard<std::mutex> g(emu);
            if (!ecode) {
                ecode = e.code;
                emsg = e.what();
            }
        } catch (const std::exception& e) {
            std::lock_guard<std::mutex> g(emu);
            if (!ecode) {
                ecode = ERR_CUDA;
                emsg = e.what();
            }
        }
    };
    const uint32_t t = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(threads ? threads : 1, n));
    std::vector<std::thread> pool;
    for (uint32_t j = 1; j < t; ++j) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    if (ecode) throw WError(ecode, emsg);
}

}  // namespace

// ===========================================================================
// C ABI
extern "C" {

const char* within_last_error(void) { return g_err.c_str(); }
uint64_t within_launch_count(void) { return g_launches; }
void within_launch_count_reset(void) { g_launches = 0; }

void within_precond_config_default(within_precond_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->kind = WITHIN_PRECOND_ADDITIVE;
    c->approx_chol_seed = 0;
    c->approx_chol_split = 2;
    c->schur_exact = 0;
    c->schur_seed = 0;
    c->schur_split = 1;
    c->dense_threshold = 24;
    c->scaling_tolerance = 1e-9;
    c->scaling_max_sweeps = 2048;
    c->scaling_error = 0;
    c->reduction = 0;
}

void within_lsmr_options_default(within_lsmr_options* o) {
    o->tol = 1e-8;
    o->maxiter = 1000;
    o->local_size = 0;
}

int within_design_from_categories(const uint32_t* codes, uint64_t n_obs, uint64_t n_factors,
                                  within_design** out) {
    *out = nullptr;
    return guarded([&] {
        if (!codes && n_obs * n_factors) throw WError(ERR_INVALID, "codes is NULL");
        if (n_obs == 0) throw WError(ERR_BUILD, "no observations provided");
        auto d = std::make_unique<within_design>();
        d->n_obs = n_obs;
        d->levels.resize(n_factors);
        d->intercept.assign(n_factors, 1);
        d->slope_of.resize(n_factors);
        // the columns copied (and their largest codes found) side by side
        std::vector<uint32_t> mx(n_factors, 0);
        par_for_each(n_factors, [&](size_t f) {
            d->levels[f].assign(codes + f * n_obs, codes + (f + 1) * n_obs);
            mx[f] = *std::max_element(d->levels[f].begin(), d->levels[f].end());
        });
        uint64_t nd = 0;
        for (uint32_t m : mx) nd += (uint64_t)m + 1;
        d->n_dofs = nd;
        *out = d.release();
    });
}

int within_design_from_effects(uint64_t n_obs, uint64_t n_effects, const uint32_t* const* levels,
                               const int32_t* intercept, const uint64_t* n_slopes,
                               const double* const* slopes, within_design** out) {
    *out = nullptr;
    return guarded([&] {
        if (n_obs == 0) throw WError(ERR_BUILD, "no observations provided");
        auto d = std::make_unique<within_design>();
        d->n_obs = n_obs;
        uint64_t si = 0;
        for (uint64_t e = 0; e < n_effects; ++e) {
            d->intercept.push_back(intercept[e] ? 1 : 0);
            std::vector<size_t> idx;
            for (uint64_t j = 0; j < n_slopes[e]; ++j, ++si) idx.push_back(si);
            if (!intercept[e] && idx.empty())
                throw WError(ERR_BUILD, "an effect must have an intercept or at least one slope");
            d->slope_of.push_back(idx);
        }
        // the level and slope columns copied (and the largest codes found) side by side
        d->levels.resize(n_effects);
        d->slopes.resize(si);
        std::vector<uint32_t> mx(n_effects, 0);
        par_for_each(n_effects + si, [&](size_t i) {
            if (i < n_effects) {
                d->levels[i].assign(levels[i], levels[i] + n_obs);
                mx[i] = *std::max_element(d->levels[i].begin(), d->levels[i].end());
            } else {
                const size_t j = i - n_effects;
                d->slopes[j].assign(slopes[j], slopes[j] + n_obs);
            }
        });
        uint64_t nd = 0;
        for (uint64_t e = 0; e < n_effects; ++e)
            nd += ((uint64_t)mx[e] + 1) * ((intercept[e] ? 1 : 0) + d->slope_of[e].size());
        d->n_dofs = nd;
        *out = d.release();
    });
}

void within_design_free(within_design* d) { delete d; }
uint64_t within_design_n_obs(const within_design* d) { return d ? d->n_obs : 0; }
uint64_t within_design_n_dofs(const within_design* d) { return d ? d->n_dofs : 0; }

int within_solver_new(const within_design* design, const double* weights, const within_precond_config* cfg,
                      const within_preconditioner* prebuilt, int32_t device, within_solver** out) {
    *out = nullptr;
    return guarded([&] { *out = make_solver(design, weights, cfg, prebuilt, device); });
}

void within_tuning_default(within_tuning* t) {
    if (!t) return;
    t->staged_sweep = 1;
    t->wide_mean_len = UINT32_MAX;
    t->fuse_rounds = 1;
    t->thread_per_segment = 1;
    PrecondCfg pc;
    t->core_dense_max = pc.core_dense_max;
    t->core_min_frac = pc.core_min_frac;
    t->max_rounds = pc.max_rounds;
    t->core_small = pc.core_small;
    t->core_dense_late = pc.core_dense_late;
    t->warp_ranges = 1;
    t->gpu_cross_tab = 1;
    t->vector_rows = 0;
}

int within_solver_new_tuned(const within_design* design, const double* weights, const within_precond_config* cfg,
                            const within_preconditioner* prebuilt, int32_t device, const within_tuning* tuning,
                            within_solver** out) {
    *out = nullptr;
    return guarded([&] {
        if (tuning && !(tuning->core_min_frac >= 0.0 && tuning->core_min_frac <= 1.0))
            throw WError(ERR_INVALID, "tuning: core_min_frac must lie in [0, 1]");
        *out = make_solver(design, weights, cfg, prebuilt, device, tuning);
    });
}

int within_solvers_new(uint64_t n, const within_design* const* designs, const double* const* weights,
                       const within_precond_config* cfg, int32_t device, uint32_t threads, within_solver** out) {
    return guarded([&] {
        for (uint64_t i = 0; i < n; ++i) out[i] = nullptr;
        int dev = device;
        if (dev < 0) CK(cudaGetDevice(&dev));
        try {
            parallel_for(n, threads, dev, [&](uint64_t i) {
                if (!designs[i]) throw WError(ERR_INVALID, "design " + std::to_string(i) + " is null");
                out[i] = make_solver(designs[i], weights ? weights[i] : nullptr, cfg, nullptr, dev, nullptr, false);
            });
        } catch (...) {
            for (uint64_t i = 0; i < n; ++i) {
                delete out[i];
                out[i] = nullptr;
            }
            throw;
        }
    });
}

int within_solvers_solve_batch(uint64_t n, within_solver* const* solvers, const double* const* Y, const uint64_t* k,
                               const within_lsmr_options* opts, double* const* X, double* const* D,
                               within_solve_stats* const* stats, uint32_t threads) {
    return guarded([&] {
        if (n == 0) return;
        parallel_for(n, threads, solvers[0]->device, [&](uint64_t i) {
            if (k[i] == 0) return;
            host_solve(*solvers[i], Y[i], k[i], opts, X ? X[i] : nullptr, D ? D[i] : nullptr,
                       stats ? stats[i] : nullptr);
        });
    });
}

void within_solver_free(within_solver* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    delete s;
}

uint64_t within_solver_n_obs(const within_solver* s) { return s->n_obs; }
uint64_t within_solver_n_dofs(const within_solver* s) { return s->n_dofs; }
uint64_t within_solver_n_warnings(const within_solver* s) { return s->n_warnings; }
uint64_t within_solver_unidentified(const within_solver* s, uint64_t* triples, uint64_t cap) {
    const auto& u = s->reparam.unidentified;
    uint64_t n = u.size() / 3;
    for (uint64_t i = 0; i < n && i < cap; ++i)
        for (int j = 0; j < 3; ++j) triples[3 * i + j] = u[3 * i + j];
    return n;
}
uint64_t within_solver_n_terms(const within_solver* s) { return s->design.terms.size(); }
int within_solver_term_layout(const within_solver* s, uint64_t term, uint64_t* n_levels, uint64_t* offset,
                              uint64_t* n_columns) {
    if (term >= s->design.terms.size()) {
        g_err = "term out of range";
        return WITHIN_ERR_INVALID_INPUT;
    }
    const Term& t = s->design.terms[term];
    *n_levels = t.n_levels;
    *offset = t.offset;
    *n_columns = t.cols.size();
    return WITHIN_OK;
}
int within_solver_obs_perm(const within_solver* s, uint32_t* out) {
    if (s->design.obs_perm.empty()) return 0;
    std::memcpy(out, s->design.obs_perm.data(), s->n_obs * sizeof(uint32_t));
    return 1;
}
within_preconditioner* within_solver_preconditioner(const within_solver* s) {
    if (!s->precond) return nullptr;
    ++s->precond->refs;
    return s->precond;
}
int within_solver_set_precision(within_solver* s, int32_t precision) {
    if (precision != WITHIN_PRECISION_FP64 && precision != WITHIN_PRECISION_MIXED) {
        g_err = "unknown precision " + std::to_string(precision);
        return WITHIN_ERR_INVALID_INPUT;
    }
    std::lock_guard<std::mutex> g(s->mu);
    s->precision = precision;
    return WITHIN_OK;
}

int within_solver_solve(within_solver* s, const double* y, const within_lsmr_options* opts, double* x_out,
                        double* demeaned_out, within_solve_stats* stats) {
    return guarded([&] { host_solve(*s, y, 1, opts, x_out, demeaned_out, stats); });
}

int within_solver_solve_batch(within_solver* s, const double* Y, uint64_t k, const within_lsmr_options* opts,
                              double* X_out, double* D_out, within_solve_stats* stats) {
    return guarded([&] {
        if (k == 0) return;
        host_solve(*s, Y, k, opts, X_out, D_out, stats);
    });
}

int within_solver_solve_batch_device(within_solver* s, const double* Y_dev, uint64_t k,
                                     const within_lsmr_options* opts, double* X_dev, double* D_dev,
                                     within_solve_stats* stats, void* stream) {
    return guarded([&] {
        double tol;
        uint64_t maxiter, ls;
        validate_opts(opts, tol, maxiter, ls);
        if (k == 0) return;
        std::lock_guard<std::mutex> g(s->mu);
        set_device(s->device);
        cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
        dispatch_solve(*s, Y_dev, k, tol, maxiter, X_dev, D_dev, stats, st, ls);
        if (X_dev && s->reparam.active()) {
            std::vector<double> hx(k * s->n_dofs);
            CK(cudaMemcpyAsync(hx.data(), X_dev, hx.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (uint64_t j = 0; j < k; ++j) s->reparam.back_transform(hx.data() + j * s->n_dofs);
            CK(cudaMemcpyAsync(X_dev, hx.data(), hx.size() * sizeof(double), cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
        }
    });
}

int within_solver_solve_batch_device_ext(within_solver* s, const double* Y_dev, uint64_t k,
                                         const within_lsmr_options* opts, const within_solve_ext* ext,
                                         double* X_dev, double* D_dev, within_solve_stats* stats,
                                         int32_t* stop_reason, void* stream) {
    return guarded([&] {
        double tol;
        uint64_t maxiter, ls;
        validate_opts(opts, tol, maxiter, ls);
        SolveExt e;
        if (ext) {
            e.x0 = ext->x0_dev;
            e.stale_window = ext->stale_window;
            e.stale_threshold = ext->stale_threshold;
            if (e.stale_window && !(e.stale_threshold >= 0.0 && e.stale_threshold < 1.0))
                throw WError(ERR_INVALID, "staleness threshold must be in [0, 1), got " +
                                              std::to_string(e.stale_threshold));
            if (e.stale_window > (uint64_t)INT_MAX) throw WError(ERR_INVALID, "staleness window too large");
        }
        if (k == 0) return;
        std::lock_guard<std::mutex> g(s->mu);
        set_device(s->device);
        if (e.x0 && s->reparam.active())
            throw WError(ERR_UNSUPPORTED, "warm starts are supported for designs without slope terms");
        cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
        dispatch_solve(*s, Y_dev, k, tol, maxiter, X_dev, D_dev, stats, st, ls, e, stop_reason);
        if (X_dev && s->reparam.active()) {
            std::vector<double> hx(k * s->n_dofs);
            CK(cudaMemcpyAsync(hx.data(), X_dev, hx.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (uint64_t j = 0; j < k; ++j) s->reparam.back_transform(hx.data() + j * s->n_dofs);
            CK(cudaMemcpyAsync(X_dev, hx.data(), hx.size() * sizeof(double), cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
        }
    });
}

int within_solve(const within_design* design, const double* y, const double* weights,
                 const within_lsmr_options* opts, const within_precond_config* cfg, double* x_out,
                 double* demeaned_out, within_solve_stats* stats) {
    return within_solve_batch(design, y, 1, weights, opts, cfg, x_out, demeaned_out, stats);
}

int within_solve_batch(const within_design* design, const double* Y, uint64_t k, const double* weights,
                       const within_lsmr_options* opts, const within_precond_config* cfg, double* X_out,
                       double* D_out, within_solve_stats* stats) {
    return guarded([&] {
        const double t0 = now_s();
        std::unique_ptr<within_solver> s(make_solver(design, weights, cfg, nullptr, -1));
        const double t1 = now_s();
        if (k == 0) return;
        host_solve(*s, Y, k, opts, X_out, D_out, stats);
        if (stats)
            for (uint64_t j = 0; j < k; ++j) {
                stats[j].time_setup += t1 - t0;
                stats[j].time_total = now_s() - t0;
            }
        cudaStreamSynchronize(s->stream);
    });
}

int within_solver_operator_apply(within_solver* s, const double* x_dev, double* y_dev, void* stream) {
    return guarded([&] {
        std::lock_guard<std::mutex> g(s->mu);
        set_device(s->device);
        cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
        if (!launch_tgather(*s, x_dev, nullptr, y_dev, false, nullptr, s->sweep_err, st)) {
            launch_k(k_apply<1>, grid_for(s->n_obs, 256, 148 * 16), 256, 0, st, s->op, x_dev, y_dev, (const int*)nullptr);
            ++g_launches;
        }
        CK(cudaGetLastError());
        if (!stream) {
            CK(cudaStreamSynchronize(st));
            int e = 0;
            CK(cudaMemcpy(&e, s->sweep_err, sizeof(int), cudaMemcpyDeviceToHost));
            if (e) throw WError(ERR_CUDA, "staged gather: a bulk copy into shared memory did not complete within 1 s");
        }
    });
}

int within_solver_operator_apply_adjoint(within_solver* s, const double* u_dev, double* y_dev, void* stream) {
    return guarded([&] {
        std::lock_guard<std::mutex> g(s->mu);
        set_device(s->device);
        cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
        ensure_scatter(*s, 1);
        const int path = env_path(2);
        if (path == 2) {
            auto& rk = ensure_rowsweep<1>(*s);
            CK(cudaMemsetAsync(y_dev, 0, s->n_dofs * sizeof(double), st));   // levels no row reaches stay 0
            launch_rowsweep<1, 0, double>(*s, rk, s->op, y_dev, nullptr, const_cast<double*>(u_dev), nullptr,
                                          nullptr, nullptr, 0, st);
            rowsweep_rest<1, double>(*s, rk, u_dev, y_dev, nullptr, st);
            CK(cudaGetLastError());
            if (!stream) {
                CK(cudaStreamSynchronize(st));
                int e = 0;
                CK(cudaMemcpy(&e, s->sweep_err, sizeof(int), cudaMemcpyDeviceToHost));
                if (e) throw WError(ERR_CUDA, "row sweep: a bulk copy into shared memory did not complete within 1 s");
            }
            return;
        }
        scatter<1, 0>(*s, u_dev, y_dev, nullptr, nullptr, st);
        CK(cudaGetLastError());
        if (!stream) CK(cudaStreamSynchronize(st));
    });
}

void within_preconditioner_free(within_preconditioner* p) {
    if (p && --p->refs == 0) delete p;
}
uint64_t within_preconditioner_n(const within_preconditioner* p) { return p ? p->n : 0; }
// ---- persisted preconditioner: the host image in this library's own byte
// format (magic, version, kind, DOF count, then every field of the diagonal
// or Schwarz image as a length-prefixed little-endian array in a fixed order,
// then an FNV-1a checksum of everything before it).  It plays the part of the
// reference's pickled Preconditioner (crates/within-py/src/config.rs:366-389,
// operator/schwarz.rs:115-183); the reference's postcard bytes embed
// approx-chol's private factor layout, so the two formats are not
// interchangeable.
}  // extern "C"
namespace {

constexpr char PC_MAGIC[8] = {'W', 'G', 'P', 'U', 'P', 'C', 'N', 'D'};
constexpr uint32_t PC_VERSION = 1;

#define WGPU_SCHWARZ_FIELDS(X)                                                                          \
    X(n_dofs) X(n_sub) X(loc_ptr) X(n_elim) X(red_off) X(n_kept) X(red_n) X(mode) X(kept_ptr) X(glob)   \
    X(scale) X(slot_sub) X(inv_e) X(ct_ptr) X(ct_col) X(ct_val) X(ct_rowsum) X(ct_row_slot)             \
    X(ct_row_red) X(elim_slot) X(c_ptr) X(c_col) X(c_val) X(n_red) X(red_sub) X(dense_rows_ptr)         \
    X(dense_row_slot) X(dense_col) X(dense_val) X(n_rounds) X(dinv) X(fwd_round_ptr) X(fwd_row)         \
    X(fwd_ptr) X(fwd_col) X(fwd_val) X(bwd_round_ptr) X(bwd_row) X(bwd_ptr) X(bwd_col) X(bwd_val)       \
    X(core_rows_ptr) X(core_row_slot) X(core_col) X(core_val) X(max_core) X(dof_ptr) X(dof_slot)        \
    X(factor_nnz) X(cross_nnz) X(max_round_rows)

uint64_t fnv1a(const uint8_t* p, size_t n) {
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

struct PcWriter {
    std::vector<uint8_t> b;
    template <class T>
    void put(const T& v) {
        static_assert(std::is_trivially_copyable<T>::value, "pod");
        const auto* q = reinterpret_cast<const uint8_t*>(&v);
        b.insert(b.end(), q, q + sizeof(T));
    }
    template <class T>
    void io(const T& v) { put(v); }
    template <class T>
    void io(const std::vector<T>& v) {
        put((uint64_t)v.size());
        const auto* q = reinterpret_cast<const uint8_t*>(v.data());
        b.insert(b.end(), q, q + v.size() * sizeof(T));
    }
};

struct PcReader {
    const uint8_t* p;
    size_t n, off = 0;
    void need(size_t k) {
        if (k > n - off) throw WError(ERR_INVALID, "preconditioner bytes are truncated");
    }
    template <class T>
    void get(T& v) {
        need(sizeof(T));
        std::memcpy(&v, p + off, sizeof(T));
        off += sizeof(T);
    }
    template <class T>
    void io(T& v) { get(v); }
    template <class T>
    void io(std::vector<T>& v) {
        uint64_t len = 0;
        get(len);
        if (len > (n - off) / sizeof(T)) throw WError(ERR_INVALID, "preconditioner bytes are truncated");
        v.resize(len);
        std::memcpy(v.data(), p + off, len * sizeof(T));
        off += len * sizeof(T);
    }
};

template <class IO, class H>
void schwarz_io(IO& io, H& h) {
#define WGPU_IO_FIELD(f) io.io(h.f);
    WGPU_SCHWARZ_FIELDS(WGPU_IO_FIELD)
#undef WGPU_IO_FIELD
}

std::vector<uint8_t> serialize_precond(const within_preconditioner& P) {
    PcWriter w;
    w.b.insert(w.b.end(), PC_MAGIC, PC_MAGIC + 8);
    w.put(PC_VERSION);
    w.put((int32_t)P.kind);
    w.put((uint32_t)P.n);
    if (P.kind == 2) w.io(P.host_inv_diag);
    else schwarz_io(w, P.host);
    w.put(fnv1a(w.b.data(), w.b.size()));
    return std::move(w.b);
}

within_preconditioner* deserialize_precond(const uint8_t* buf, size_t len, int device) {
    if (!buf || len < 8 + 4 + 4 + 4 + 8) throw WError(ERR_INVALID, "preconditioner bytes are truncated");
    if (std::memcmp(buf, PC_MAGIC, 8) != 0) throw WError(ERR_INVALID, "not a serialised within_b200 preconditioner");
    uint64_t sum = 0;
    std::memcpy(&sum, buf + len - 8, 8);
    if (sum != fnv1a(buf, len - 8)) throw WError(ERR_INVALID, "preconditioner bytes are corrupt (checksum)");
    PcReader r{buf, len - 8, 8};
    uint32_t ver = 0, n = 0;
    int32_t kind = 0;
    r.get(ver);
    if (ver != PC_VERSION)
        throw WError(ERR_UNSUPPORTED, "preconditioner format version " + std::to_string(ver) + " (this build reads " +
                                          std::to_string(PC_VERSION) + ")");
    r.get(kind);
    r.get(n);
    if (kind != 1 && kind != 2) throw WError(ERR_INVALID, "preconditioner bytes hold an unknown kind");
    if (device < 0) CK(cudaGetDevice(&device));
    set_device(device);
    auto P = std::make_unique<within_preconditioner>();
    P->device = device;
    P->kind = kind;
    P->n = n;
    if (kind == 2) {
        r.io(P->host_inv_diag);
        if (P->host_inv_diag.size() != n) throw WError(ERR_INVALID, "preconditioner bytes: diagonal size mismatch");
        P->inv_diag = P->arena.upload(P->host_inv_diag);
    } else {
        SchwarzHost H;
        schwarz_io(r, H);
        if (H.n_dofs != n) throw WError(ERR_INVALID, "preconditioner bytes: DOF count mismatch");
        upload_schwarz(*P, std::move(H));
    }
    if (r.off != r.n) throw WError(ERR_INVALID, "preconditioner bytes have trailing data");
    CK(cudaDeviceSynchronize());
    return P.release();
}

}  // namespace
extern "C" {

int within_preconditioner_serialize(const within_preconditioner* p, uint8_t* buf, uint64_t cap, uint64_t* len) {
    return guarded([&] {
        if (!p || !len) throw WError(ERR_INVALID, "within_preconditioner_serialize: NULL argument");
        std::lock_guard<std::mutex> g(const_cast<within_preconditioner*>(p)->mu);
        const std::vector<uint8_t> b = serialize_precond(*p);
        *len = b.size();
        if (!buf) return;
        if (cap < b.size())
            throw WError(ERR_INVALID, "within_preconditioner_serialize: buffer of " + std::to_string(cap) +
                                          " bytes, " + std::to_string(b.size()) + " needed");
        std::memcpy(buf, b.data(), b.size());
    });
}

int within_preconditioner_deserialize(const uint8_t* buf, uint64_t len, int32_t device,
                                      within_preconditioner** out) {
    return guarded([&] {
        if (!out) throw WError(ERR_INVALID, "within_preconditioner_deserialize: NULL output");
        *out = nullptr;
        *out = deserialize_precond(buf, (size_t)len, device);
    });
}

int within_preconditioner_stats(const within_preconditioner* p, within_precond_stats* out) {
    return guarded([&] {
        if (!p || !out) throw WError(ERR_INVALID, "within_preconditioner_stats: NULL argument");
        *out = within_precond_stats{};
        out->n = p->n;
        if (p->kind != 1) return;
        const SchwarzHost& H = p->host;
        out->n_subdomains = H.n_sub;
        out->n_slots = H.glob.size();
        out->nnz_c = H.c_col.size();
        out->nnz_ct = H.ct_col.size();
        out->nnz_fwd = H.fwd_col.size();
        out->nnz_bwd = H.bwd_col.size();
        out->nnz_dense = H.dense_col.size();
        out->nnz_core = H.core_col.size();
        out->n_reduced = H.n_red;
        out->n_rounds = H.n_rounds;
    });
}
const char* within_preconditioner_variant_name(const within_preconditioner* p) {
    return p && p->kind == 2 ? "Diagonal" : "Additive";
}

int within_preconditioner_apply(const within_preconditioner* pc, const double* x_dev, double* y_dev,
                                void* stream) {
    return guarded([&] {
        auto* p = const_cast<within_preconditioner*>(pc);
        set_device(p->device);
        cudaStream_t st = stream ? (cudaStream_t)stream : nullptr;
        if (p->kind == 2) {
            launch_k(k_diag_apply<1>, grid_for(p->n, 256, 148 * 8), 256, 0, st, p->n, p->inv_diag, x_dev, y_dev, nullptr);
            ++g_launches;
        } else {
            std::lock_guard<std::mutex> g(p->mu);
            if (!p->standalone) {
                p->standalone = new SchwarzUser();
                p->standalone->tuning = resolve_tuning(nullptr);
            }
            schwarz_apply<1>(*p, *p->standalone, x_dev, y_dev, nullptr, st);
        }
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
    });
}

int within_adjoint_rhs(uint64_t n, uint64_t k, const double* v_dev, const double* w_dev, double* a_dev,
                       void* stream) {
    return guarded([&] {
        if (n == 0 || k == 0) return;
        if (!v_dev || !a_dev) throw WError(ERR_INVALID, "adjoint rhs: null buffer");
        cudaStream_t st = (cudaStream_t)stream;
        launch_k(k_adjoint_rhs, grid_for(n, 256, 148 * 16), 256, 0, st, n, (uint32_t)k, v_dev, w_dev, a_dev);
        ++g_launches;
        CK(cudaGetLastError());
    });
}

int within_demean_vjp(uint64_t n, uint64_t k, const double* r_dev, const double* a_dev, const double* s_dev,
                      const double* w_dev, double* grad_z_dev, double* grad_w_dev, void* stream) {
    return guarded([&] {
        if (n == 0 || k == 0) return;
        if (!s_dev || (grad_w_dev && (!r_dev || !a_dev)))
            throw WError(ERR_INVALID, "demean vjp: null buffer");
        cudaStream_t st = (cudaStream_t)stream;
        launch_k(k_demean_vjp, grid_for(n, 256, 148 * 16), 256, 0, st, n, (uint32_t)k, r_dev, a_dev, s_dev, w_dev,
                                                                  grad_z_dev, grad_w_dev);
        ++g_launches;
        CK(cudaGetLastError());
    });
}

}  // extern "C"

// ===========================================================================
// Allocation-free variant of within_solver_operator_apply_adjoint.
//
// Some callers cannot allocate device memory while they run: code executing
// under a CUDA stream capture (allocations are not capturable), runtimes that
// own all device memory through their own arena and forbid cudaMalloc from
// libraries, and real-time paths where an allocation's implicit
// synchronisation or failure is unacceptable.  This entry point computes the
// same D^T (W^{1/2} u) as within_solver_operator_apply_adjoint, but the
// segmented reduction's scratch -- the per-tile partial sums and the per-split
// completion counters -- lives in the file-scope device array below instead of
// solver-owned allocations, and nothing is allocated during the call.
namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)8 << 20;   // 8 MiB
// Present on every device that loads this library, for the process lifetime.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_dev_ptr[NOALLOC_MAX_DEVICES] = {};

// Device address of g_noalloc_scratch on `dev` (which must be current).  On the
// host the array's name only identifies the symbol; the address is looked up
// on every call outside stream capture (so a context created after a device
// reset gets its own) and the last one is reused while `st` is capturing.
void* noalloc_scratch(int dev, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) throw WError(ERR_UNSUPPORTED, "device ordinal out of range");
    if (cs == cudaStreamCaptureStatusNone || !g_noalloc_dev_ptr[dev]) {
        void* p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_dev_ptr[dev] = p;
    }
    return g_noalloc_dev_ptr[dev];
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" int within_solver_operator_apply_adjoint_noalloc(within_solver* s, const double* u_dev,
                                                            double* y_dev, void* stream) {
    return guarded([&] {
        if (!s) throw WError(ERR_INVALID, "solver is NULL");
        std::lock_guard<std::mutex> g(s->mu);
        set_device(s->device);
        if (!s->scatter_ready[0])
            throw WError(ERR_INVALID,
                         "within_solver_operator_apply_adjoint_noalloc: the solver's single-column tile plan "
                         "is missing (it is built at construction)");
        const DevPlan& pl = s->scatter_plan[0];
        const size_t head_b = align256((size_t)pl.n_tiles * sizeof(double));
        const size_t tail_b = align256((size_t)std::max<uint32_t>(1, pl.n_splits) * sizeof(double));
        const size_t cnt_b = align256((size_t)std::max<uint32_t>(1, pl.n_splits) * sizeof(unsigned));
        const size_t need = head_b + tail_b + cnt_b;
        if (need > NOALLOC_SCRATCH_BYTES)
            throw WError(ERR_UNSUPPORTED,
                         "within_solver_operator_apply_adjoint_noalloc: this design needs " + std::to_string(need) +
                         " bytes of scratch (" + std::to_string(pl.n_tiles) + " tiles, " +
                         std::to_string(pl.n_splits) + " split segments); the static maximum is " +
                         std::to_string(NOALLOC_SCRATCH_BYTES) + " bytes");
        cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
        char* base = (char*)noalloc_scratch(s->device, st);
        DevPlan p = pl;
        p.head = (double*)base;
        p.tail = (double*)(base + head_b);
        p.counters = (unsigned*)(base + head_b + tail_b);
        // the completion counters must start at zero; partials are written before they are read
        CK(cudaMemsetAsync(p.counters, 0, cnt_b, st));
        ScatterF<1, 0> f{s->scatter_probs, u_dev, s->op.sqrt_w, y_dev, nullptr};
        launch_sr<ScatterF<1, 0>, 1>(f, p, 0, p.n_tiles, nullptr, st);
        CK(cudaGetLastError());
        if (!stream) CK(cudaStreamSynchronize(st));
    });
}
