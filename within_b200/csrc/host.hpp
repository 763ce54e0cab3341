// host.hpp -- host-side set-up of the B200 fixed-effects solver: design
// layout, slope reparametrisation, preconditioner construction and the tile
// plans of the segmented-reduction engine.  Runs once per Solver; everything
// it produces is uploaded and stays resident in HBM across solves.
#pragma once
#include <cstdint>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <future>
#include <vector>

#include "segplan.hpp"

namespace wgpu {

struct WError : std::runtime_error {
    int code;
    WError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
enum { ERR_INVALID = 1, ERR_BUILD = 2, ERR_UNSCALABLE = 3, ERR_SINGULAR = 4, ERR_INDEFINITE = 5,
       ERR_DIMENSION = 6, ERR_CUDA = 7, ERR_UNSUPPORTED = 8 };

constexpr int MAX_TERMS = 8;
constexpr int MAX_COLS = 4;     // coefficient columns per term (intercept + slopes)
constexpr int MAX_LOADS = 16;   // slope columns in a design

// One term's layout: coefficient c of level l sits at offset + c*n_levels + l
// (crates/within/src/domain.rs:79-103).  cols[c] = -1 for the intercept,
// otherwise the loading column index.
struct Term {
    uint32_t n_levels = 0, offset = 0;
    bool sorted = true;
    std::vector<int> cols;
    uint32_t n_dofs() const { return (uint32_t)(cols.size() * n_levels); }
};

struct HostDesign {
    uint64_t n_obs = 0, n_dofs = 0;
    std::vector<Term> terms;
    std::vector<std::vector<uint32_t>> codes;   // per term, internal order
    std::vector<std::vector<double>> loads;     // per loading column, internal order
    std::vector<uint32_t> obs_perm;             // internal -> caller; empty = identity
};

// Effect description as handed over the C ABI.
struct EffectIn {
    const uint32_t* levels;
    bool intercept;
    std::vector<const double*> slopes;
};
HostDesign make_design(uint64_t n_obs, const std::vector<EffectIn>& effects);
void stable_argsort_u32(const uint32_t* key, size_t n, size_t n_levels, uint32_t* perm);

// Within-level whitening of slope columns (crates/within/src/solver/reparam.rs).
struct Reparam {
    struct TermR {
        uint32_t offset = 0, n_levels = 0;
        int intercept_col = -1;
        std::vector<uint32_t> slope_cols;
        // per level: w (rank x V row-major, rank = rows present) and center (V)
        std::vector<std::vector<double>> w, center;
    };
    std::vector<TermR> terms;
    std::vector<uint64_t> unidentified;   // (term, level, column) triples
    bool active() const { return !terms.empty(); }
    void back_transform(double* x) const;
};
Reparam build_reparam(HostDesign& d, const double* weights_internal);

// ---- preconditioner configuration (crates/within/src/config.rs:61-157) ----
struct PrecondCfg {
    int kind = 1;  // 0 off, 1 additive, 2 diagonal
    uint64_t ac_seed = 0;
    uint32_t ac_split = 2;
    bool schur_exact = false;
    uint64_t schur_seed = 0;
    uint32_t schur_split = 1;
    uint64_t dense_threshold = 24;
    double scaling_tol = 1e-9;
    uint64_t scaling_max_sweeps = 2048;
    bool scaling_error = false;
    // round-parallel factor: when to stop the rounds (host_schwarz.cpp ac_rounds)
    uint32_t core_dense_max = 2048;   // a reduced system this small is inverted densely at once
    double core_min_frac = 0.3;       // a large graph stops when a round eliminates less than this
    uint32_t max_rounds = 64;
    uint32_t core_small = 16384;      // at or below: rounds continue past core_min_frac ...
    uint32_t core_dense_late = 512;   // ... until this many vertices remain (dense core)
    double core_min_frac_small = 0.005;   // (or a round eliminates less than this)
};

// Host image of the additive Schwarz preconditioner in the layout the apply
// kernels read.  All subdomains are concatenated: local slots (eliminated
// block first, then kept block) for the restrict/prolong side, and reduced
// slots for the reduced triangular solves.
struct SchwarzHost {
    uint32_t n_dofs = 0;
    uint32_t n_sub = 0;
    // per subdomain
    std::vector<uint32_t> loc_ptr;        // n_sub+1 local-slot ranges
    std::vector<uint32_t> n_elim;         // eliminated block size
    std::vector<uint32_t> red_off;        // first reduced slot
    std::vector<uint32_t> n_kept;         // kept block size
    std::vector<uint32_t> red_n;          // reduced system size (factor dimension)
    std::vector<int32_t> mode;            // 0 floating, 1 grounded (explicit ground at kept), 2 cover
    std::vector<uint32_t> kept_ptr;       // n_sub+1 ranges over the concatenated kept rows
    // per local slot
    std::vector<uint32_t> glob;           // global DOF
    std::vector<double> scale;            // partition weight * coordinate factor
    std::vector<uint32_t> slot_sub;       // owning subdomain
    std::vector<double> inv_e;            // 1/D_e for eliminated slots (0 for kept)
    // C^T rows: one per kept slot, columns = local slot of the eliminated entry,
    // values C^T[k,e] / D_e[e]; ct_rowsum[k] = sum of the row's values
    std::vector<uint32_t> ct_ptr, ct_col;
    std::vector<double> ct_val, ct_rowsum;
    std::vector<uint32_t> ct_row_slot;    // kept local slot of each C^T row
    std::vector<uint32_t> ct_row_red;     // reduced slot of each C^T row
    // C rows: one per eliminated slot (in local-slot order of eliminated slots)
    std::vector<uint32_t> elim_slot;      // local slot of each C row
    // columns = reduced slot of the kept entry (bit 31 set when the kept
    // solution needs the ground gauge or the cover read-back); values C[e,k] / D_e[e]
    std::vector<uint32_t> c_ptr, c_col;
    std::vector<double> c_val;
    // reduced slots
    uint32_t n_red = 0;
    std::vector<uint32_t> red_sub;        // owning subdomain of each reduced slot
    // dense pseudo-inverse blocks (small reduced systems): row-major per subdomain
    std::vector<uint32_t> dense_rows_ptr; // segments = reduced rows of dense subdomains
    std::vector<uint32_t> dense_row_slot; // reduced slot of each dense row
    std::vector<uint32_t> dense_col;      // reduced slot of each entry
    std::vector<double> dense_val;
    // level-scheduled approximate-Cholesky factors (L D L^T, unit lower L)
    uint32_t n_rounds = 0;
    std::vector<double> dinv;             // per reduced slot, 1/pivot (0 = null pivot)
    std::vector<uint32_t> fwd_round_ptr;  // n_rounds+1 over fwd rows
    std::vector<uint32_t> fwd_row;        // reduced slot of each row, grouped by round
    std::vector<uint32_t> fwd_ptr, fwd_col;   // pull form: L[row, col] for earlier cols
    std::vector<double> fwd_val;
    std::vector<uint32_t> bwd_round_ptr;  // n_rounds+1 (round r listed in elimination order)
    std::vector<uint32_t> bwd_row;
    std::vector<uint32_t> bwd_ptr, bwd_col;   // pull form: L[later row, col]
    std::vector<double> bwd_val;
    // dense cores of round-scheduled factors (x_core = G y_core after the forward pass)
    std::vector<uint32_t> core_rows_ptr, core_row_slot, core_col;
    std::vector<double> core_val;
    uint32_t max_core = 0;
    // prolongation combine: DOF -> local slots
    std::vector<uint32_t> dof_ptr, dof_slot;
    // statistics
    uint64_t factor_nnz = 0, cross_nnz = 0;
    uint32_t max_round_rows = 0;
};

struct BuildResult {
    int kind = 0;                  // 0 none (unpreconditioned), 1 additive, 2 diagonal
    std::vector<double> inv_diag;  // diagonal variant
    SchwarzHost schwarz;
    uint64_t n_warnings = 0;
};
// Weighted cross-tab of one channel pair (term a column ca, term b column cb)
// over raw level ids, as computed on the GPU (xtab.cu): every cell
// (level of a, level of b) with a non-zero sum of w_i * load_a_i * load_b_i
// over its observations, each sum taken in observation order; CSR by a
// (cells of a row in ascending b) and the same cells CSC by b.
struct CrossTab {
    std::vector<uint32_t> row_ptr, col;   // L_a + 1, nnz
    std::vector<double> val;
    std::vector<uint32_t> col_ptr, row;   // L_b + 1, nnz
    std::vector<double> tval;
    // connected components of the bipartite cell graph (vertices: levels of a
    // as 0 .. L_a - 1, then levels of b as L_a .. L_a + L_b - 1): the smallest
    // vertex of each vertex's component; empty = not computed
    std::vector<uint32_t> comp;
};
// The channel pairs of a design's additive-Schwarz build, in build order:
// (term, column) of the first and second channel; columns are -1 for the
// intercept, else the slope index into HostDesign::loads.
struct ChannelPair {
    uint32_t term_a, term_b;
    int load_a, load_b;
};
std::vector<ChannelPair> schwarz_channel_pairs(const HostDesign& d);

// cross_tabs: the GPU cross-tab of every channel pair (schwarz_channel_pairs
// order; the build may move their arrays out), or nullptr to accumulate them
// on the host; both give the same bits.  ready (with cross_tabs): one future
// per pair, ready when that pair's cross-tab is filled in (its exception is
// the build's), so a pair starts as soon as its own cross-tab is back.
BuildResult build_preconditioner(const HostDesign& d, const double* weights_internal,
                                 const PrecondCfg& cfg, std::vector<CrossTab>* cross_tabs = nullptr,
                                 const std::vector<std::shared_future<void>>* ready = nullptr);

// ---- segmented-reduction plans ----
struct HostPlan {
    std::vector<SRTile> tiles;
    std::vector<SRSplit> splits;
    void add(uint32_t problem, const uint32_t* ptr, uint32_t n_seg, int tile);
};

// Range plan of the warp-range segmented sweep (segsweep.cuh): ranges of
// `range_len` positions (a multiple of SS_ALIGN), the segment-start bitmap,
// the ids of non-empty segments of problems that have empty ones, the empty
// segments (emitted as zeros by the range holding their position) and the
// split segments (positions in more than one range).
struct SSHostPlan {
    std::vector<SSRange> ranges;
    std::vector<SSSplit> splits;
    std::vector<uint32_t> bits;
    std::vector<uint32_t> nz_ids;
    std::vector<uint32_t> empties;
    void add(uint32_t problem, const uint32_t* ptr, uint32_t n_seg, uint32_t range_len);
};
// range length for `positions` positions spread over about `warps` warps
uint32_t ss_range_len(uint64_t positions, uint32_t warps);

// dense generalised inverse of a symmetric PSD matrix (the preconditioner's dense route)
std::vector<double> dense_pseudo_inverse(uint32_t n, const std::vector<double>& a);

}  // namespace wgpu
