// The additive-Schwarz build from precomputed cross-tabs (the form the GPU
// cross-tab of xtab.cu returns) against the build that accumulates them on
// the host: random designs -- unweighted intercepts, weights with zeros, a
// slope column, unused levels -- get cross-tabs made here by the GPU
// algorithm's steps (a stable sort of the (a, b) keys, per-cell sums in
// observation order, exact-zero cells dropped, CSR by a and CSC by b), and
// every array of the two host images must be bitwise equal.
#include "host.hpp"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <chrono>
#include <future>
#include <thread>
using namespace wgpu;

static CrossTab cross_tab_like_gpu(const HostDesign& d, const double* w, const ChannelPair& cp) {
    const uint64_t n = d.n_obs;
    const uint32_t La = d.terms[cp.term_a].n_levels, Lb = d.terms[cp.term_b].n_levels;
    const uint32_t* a = d.codes[cp.term_a].data();
    const uint32_t* b = d.codes[cp.term_b].data();
    const double* la = cp.load_a < 0 ? nullptr : d.loads[cp.load_a].data();
    const double* lb = cp.load_b < 0 ? nullptr : d.loads[cp.load_b].data();
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) {
        return a[x] != a[y] ? a[x] < a[y] : b[x] < b[y];
    });
    CrossTab X;
    X.row_ptr.assign(La + 1, 0);
    X.col_ptr.assign(Lb + 1, 0);
    std::vector<uint32_t> ra;
    for (size_t p = 0; p < n;) {
        size_t q = p;
        double v = 0.0;
        while (q < n && a[idx[q]] == a[idx[p]] && b[idx[q]] == b[idx[p]]) {
            const uint32_t i = idx[q];
            const double wi = w ? w[i] : 1.0, x = la ? la[i] : 1.0, y = lb ? lb[i] : 1.0;
            v += wi * x * y;
            ++q;
        }
        if (v != 0.0) {
            ra.push_back(a[idx[p]]);
            X.col.push_back(b[idx[p]]);
            X.val.push_back(v);
        }
        p = q;
    }
    for (uint32_t r : ra) ++X.row_ptr[r + 1];
    for (uint32_t r = 0; r < La; ++r) X.row_ptr[r + 1] += X.row_ptr[r];
    std::vector<uint32_t> ord(X.col.size());
    std::iota(ord.begin(), ord.end(), 0u);
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) {
        return X.col[x] != X.col[y] ? X.col[x] < X.col[y] : ra[x] < ra[y];
    });
    for (uint32_t k : ord) {
        X.row.push_back(ra[k]);
        X.tval.push_back(X.val[k]);
        ++X.col_ptr[X.col[k] + 1];
    }
    for (uint32_t c = 0; c < Lb; ++c) X.col_ptr[c + 1] += X.col_ptr[c];
    // components: the smallest vertex (levels of a, then L_a + levels of b) of each
    std::vector<uint32_t> par(La + Lb);
    std::iota(par.begin(), par.end(), 0u);
    auto find = [&](uint32_t v) {
        while (par[v] != v) v = par[v] = par[par[v]];
        return v;
    };
    for (size_t k = 0; k < ra.size(); ++k) {
        uint32_t x = find(ra[k]), y = find(La + X.col[k]);
        if (x != y) par[std::max(x, y)] = std::min(x, y);
    }
    X.comp.resize(La + Lb);
    for (uint32_t v = 0; v < La + Lb; ++v) X.comp[v] = find(v);
    return X;
}

template <class T>
static bool same(const std::vector<T>& x, const std::vector<T>& y) {
    return x.size() == y.size() && (x.empty() || std::memcmp(x.data(), y.data(), x.size() * sizeof(T)) == 0);
}

static bool same_host(const SchwarzHost& p, const SchwarzHost& q) {
#define SAME(f)                                      \
    if (!same(p.f, q.f)) {                           \
        printf("field %s differs\n", #f);            \
        return false;                                \
    }
    SAME(loc_ptr) SAME(n_elim) SAME(red_off) SAME(n_kept) SAME(red_n) SAME(mode) SAME(kept_ptr) SAME(glob)
    SAME(scale) SAME(slot_sub) SAME(inv_e) SAME(ct_ptr) SAME(ct_col) SAME(ct_val) SAME(ct_rowsum)
    SAME(ct_row_slot) SAME(ct_row_red) SAME(elim_slot) SAME(c_ptr) SAME(c_col) SAME(c_val) SAME(red_sub)
    SAME(dense_rows_ptr) SAME(dense_row_slot) SAME(dense_col) SAME(dense_val) SAME(dinv) SAME(fwd_round_ptr)
    SAME(fwd_row) SAME(fwd_ptr) SAME(fwd_col) SAME(fwd_val) SAME(bwd_round_ptr) SAME(bwd_row) SAME(bwd_ptr)
    SAME(bwd_col) SAME(bwd_val) SAME(core_rows_ptr) SAME(core_row_slot) SAME(core_col) SAME(core_val)
    SAME(dof_ptr) SAME(dof_slot)
#undef SAME
    return p.n_dofs == q.n_dofs && p.n_sub == q.n_sub && p.n_red == q.n_red && p.n_rounds == q.n_rounds &&
           p.max_core == q.max_core;
}

int main() {
    std::mt19937_64 rng(5);
    int cases = 0;
    for (int trial = 0; trial < 24; ++trial) {
        const bool big = trial % 6 == 5;   // a kept block above the dense limits: round factors
        const uint64_t n = big ? 80000 : 2000 + rng() % 30000;
        const uint32_t L0 = big ? 20000 : 50 + (uint32_t)(rng() % 3000);
        const uint32_t L1 = big ? 3000 : 5 + (uint32_t)(rng() % 400);
        const uint32_t L2 = 2 + (uint32_t)(rng() % 12);
        std::vector<uint32_t> c0(n), c1(n), c2(n);
        std::vector<double> z(n), wv(n);
        for (uint64_t i = 0; i < n; ++i) {
            c0[i] = (uint32_t)(rng() % L0) * (trial % 4 == 3 ? 2u : 1u);   // every other level unused
            c1[i] = (uint32_t)(rng() % L1);
            c2[i] = (uint32_t)(rng() % L2);
            z[i] = (double)(int64_t)(rng() % 2001) / 250.0 - 4.0;
            wv[i] = (rng() % 7 == 0) ? 0.0 : std::exp((double)(int64_t)(rng() % 2001) / 1000.0 - 1.0);
        }
        const bool weighted = trial % 2 == 1, slopes = trial % 3 == 2;
        std::vector<EffectIn> effs(3);
        effs[0].levels = c0.data();
        effs[0].intercept = true;
        effs[1].levels = c1.data();
        effs[1].intercept = true;
        if (slopes) effs[1].slopes.push_back(z.data());
        effs[2].levels = c2.data();
        effs[2].intercept = true;
        HostDesign d = make_design(n, effs);
        std::vector<double> w;
        if (weighted) {
            w.resize(n);
            for (uint64_t i = 0; i < n; ++i) w[i] = d.obs_perm.empty() ? wv[i] : wv[d.obs_perm[i]];
        }
        const double* wp = weighted ? w.data() : nullptr;
        PrecondCfg cfg;
        if (trial % 5 == 4) cfg.dense_threshold = 8;   // sampled Schur complements and round factors
        std::vector<CrossTab> xt;
        for (const ChannelPair& cp : schwarz_channel_pairs(d)) xt.push_back(cross_tab_like_gpu(d, wp, cp));
        std::vector<CrossTab> xt2 = xt;   // for the hand-over through per-pair futures below
        BuildResult host = build_preconditioner(d, wp, cfg, nullptr);
        BuildResult pre = build_preconditioner(d, wp, cfg, &xt);
        if (host.kind != pre.kind || host.n_warnings != pre.n_warnings || !same_host(host.schwarz, pre.schwarz)) {
            printf("FAIL trial %d (weighted %d slopes %d)\n", trial, (int)weighted, (int)slopes);
            return 1;
        }
        // the cross-tabs handed over one pair at a time, in reverse order and late,
        // through the per-pair futures: the same image
        {
            std::vector<CrossTab> late(xt2.size());
            std::vector<std::promise<void>> done(xt2.size());
            std::vector<std::shared_future<void>> ready;
            for (auto& p : done) ready.push_back(p.get_future().share());
            std::thread feeder([&] {
                for (size_t i = xt2.size(); i-- > 0;) {
                    std::this_thread::sleep_for(std::chrono::milliseconds(2));
                    late[i] = std::move(xt2[i]);
                    done[i].set_value();
                }
            });
            BuildResult fut = build_preconditioner(d, wp, cfg, &late, &ready);
            feeder.join();
            if (fut.kind != host.kind || fut.n_warnings != host.n_warnings || !same_host(host.schwarz, fut.schwarz)) {
                printf("FAIL trial %d (futures)\n", trial);
                return 1;
            }
        }
        ++cases;
    }
    printf("xtab ok %d\n", cases);
}
