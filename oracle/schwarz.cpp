// schwarz.cpp -- Off / Diagonal / Additive-Schwarz preconditioners restated
// from crates/within/src/{operator/schwarz.rs, domain/cross_tab*,
// domain/factor_pairs*, block_elim/*, csr_block.rs} and
// crates/schwarz-precond/src/{domain.rs, local_solve.rs, schwarz/*}.
// Sequential FP64, subdomains summed in order (the single-thread reference).
// TEST INFRASTRUCTURE ONLY.
#include "oracle_core.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <numeric>

namespace orc {

// ---------------------------------------------------------------------------
// csr_block.rs -- rectangular CSR with ascending columns.
struct Csr {
    std::vector<uint32_t> indptr{0}, indices;
    std::vector<double> data;
    size_t nrows = 0, ncols = 0;
    size_t nnz() const { return data.size(); }
};

static Csr transpose(const Csr& a) {  // csr_block.rs:58-90
    Csr t;
    t.nrows = a.ncols;
    t.ncols = a.nrows;
    t.indptr.assign(a.ncols + 1, 0);
    for (uint32_t c : a.indices) t.indptr[c + 1] += 1;
    for (size_t i = 0; i < a.ncols; ++i) t.indptr[i + 1] += t.indptr[i];
    std::vector<uint32_t> cur(t.indptr.begin(), t.indptr.end() - 1);
    t.indices.resize(a.nnz());
    t.data.resize(a.nnz());
    for (size_t r = 0; r < a.nrows; ++r)
        for (uint32_t k = a.indptr[r]; k < a.indptr[r + 1]; ++k) {
            uint32_t pos = cur[a.indices[k]]++;
            t.indices[pos] = (uint32_t)r;
            t.data[pos] = a.data[k];
        }
    return t;
}

// y = base + A x (csr_block.rs:174-190, sequential order)
static void spmv_assign_add(const Csr& a, const double* x, const double* base, double* y) {
    par_ranges(a.nrows, 8192, [&](size_t lo, size_t hi, int) {
        for (size_t i = lo; i < hi; ++i) {
            double acc = base[i];
            for (uint32_t k = a.indptr[i]; k < a.indptr[i + 1]; ++k) acc += a.data[k] * x[a.indices[k]];
            y[i] = acc;
        }
    });
}

struct CrossTab {  // cross_tab.rs:100-107
    Csr c, ct;
    size_t n_rows() const { return c.nrows; }
    size_t n_cols() const { return c.ncols; }
    size_t n_local() const { return c.nrows + c.ncols; }
    template <class F>
    void neighbors(size_t i, F f) const {  // cross_tab.rs:164-172
        size_t nr = n_rows();
        if (i < nr) {
            for (uint32_t k = c.indptr[i]; k < c.indptr[i + 1]; ++k) f(nr + c.indices[k], c.data[k]);
        } else {
            size_t r = i - nr;
            for (uint32_t k = ct.indptr[r]; k < ct.indptr[r + 1]; ++k) f((size_t)ct.indices[k], ct.data[k]);
        }
    }
};

// ---------------------------------------------------------------------------
// Diagonal preconditioner -- operator/schwarz.rs:185-229, apply 64-81.
struct DiagonalPrecond : Preconditioner {
    std::vector<double> inv;
    void apply(const double* x, double* y) const override {
        for (size_t i = 0; i < n; ++i) y[i] = inv[i] * x[i];
    }
};

static DiagonalPrecond* build_diagonal(const Design& d, const double* weights) {
    auto* p = new DiagonalPrecond();
    p->n = d.n_dofs;
    p->inv.assign(d.n_dofs, 0.0);
    for (size_t q = 0; q < d.terms.size(); ++q) {
        const auto& t = d.terms[q];
        const uint32_t* lv = d.codes[q].data();
        for (size_t c = 0; c < t.columns.size(); ++c) {
            double* slice = &p->inv[t.column_base(c)];
            int k = t.columns[c];
            for (size_t i = 0; i < d.n_obs; ++i) {
                double w = weights ? weights[i] : 1.0;
                if (k < 0)
                    slice[lv[i]] += w;
                else
                    slice[lv[i]] += w * d.loads[k][i] * d.loads[k][i];
            }
        }
    }
    for (size_t i = 0; i < d.n_dofs; ++i) {
        double& v = p->inv[i];
        if (v == 0.0) continue;
        double inv = 1.0 / v;
        if (!std::isfinite(inv)) {
            delete p;
            throw Error(E_SINGULAR, "zero diagonal in preconditioner at index " + std::to_string(i));
        }
        v = inv;
    }
    return p;
}

// ---------------------------------------------------------------------------
// Reduced-system factors (block_elim/factor.rs and the approx-chol backends).
//
// The input is always an explicit Laplacian (row sums zero; a grounded
// system carries an explicit ground vertex), as produced by
// schur::build_explicit_laplacian / build_laplacian_csr.
struct SqCsr {  // block_elim/csr_matrix.rs
    std::vector<uint32_t> indptr{0}, indices;
    std::vector<double> data;
    size_t n = 0;
};

struct Factor {
    // L D L^T with unit-lower L stored by elimination column.
    size_t n = 0;
    std::vector<uint32_t> order;             // elimination order
    std::vector<double> pivot;               // D (0 => pseudo-inverse 0), per vertex
    std::vector<uint32_t> colptr, rowidx;    // per elimination step k
    std::vector<double> val;
    void solve_in_place(double* x) const {
        for (size_t k = 0; k < n; ++k) {
            uint32_t v = order[k];
            double xv = x[v];
            for (uint32_t e = colptr[k]; e < colptr[k + 1]; ++e) x[rowidx[e]] -= val[e] * xv;
        }
        for (size_t v = 0; v < n; ++v) x[v] = pivot[v] > 0.0 ? x[v] / pivot[v] : 0.0;
        for (size_t k = n; k-- > 0;) {
            uint32_t v = order[k];
            double acc = x[v];
            for (uint32_t e = colptr[k]; e < colptr[k + 1]; ++e) acc -= val[e] * x[rowidx[e]];
            x[v] = acc;
        }
    }
};

// Dense exact backend (approx-chol Backend::ExactBelow): LDL^T in natural
// order; a pivot at or below a roundoff floor is a zero pivot (the Laplacian's
// null direction), any clearly negative pivot is a failure.
static bool dense_factor(const SqCsr& m, Factor& f) {
    const size_t n = m.n;
    std::vector<double> a(n * n, 0.0);
    double maxd = 0.0;
    for (size_t i = 0; i < n; ++i)
        for (uint32_t k = m.indptr[i]; k < m.indptr[i + 1]; ++k) {
            a[i * n + m.indices[k]] += m.data[k];
            if (m.indices[k] == i) maxd = std::max(maxd, std::fabs(m.data[k]));
        }
    const double floor = 1e-13 * std::max(maxd, DBL_MIN) * (double)std::max<size_t>(n, 1);
    f.n = n;
    f.order.resize(n);
    f.pivot.assign(n, 0.0);
    f.colptr.assign(1, 0);
    f.rowidx.clear();
    f.val.clear();
    for (size_t k = 0; k < n; ++k) {
        f.order[k] = (uint32_t)k;
        double d = a[k * n + k];
        if (d < -floor) return false;
        if (d <= floor) {
            f.pivot[k] = 0.0;
            f.colptr.push_back((uint32_t)f.rowidx.size());
            continue;
        }
        f.pivot[k] = d;
        for (size_t i = k + 1; i < n; ++i) {
            double l = a[i * n + k] / d;
            if (l != 0.0) {
                f.rowidx.push_back((uint32_t)i);
                f.val.push_back(l);
            }
        }
        for (size_t i = k + 1; i < n; ++i) {
            double lik = a[i * n + k];
            if (lik == 0.0) continue;
            for (size_t j = k + 1; j < n; ++j) a[i * n + j] -= lik * a[k * n + j] / d;
        }
        f.colptr.push_back((uint32_t)f.rowidx.size());
    }
    return true;
}

// splitmix64 stream, seeded per (seed, vertex).
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};
static uint64_t mix(uint64_t a, uint64_t b) {
    Rng r(a ^ (b * 0xD1B54A32D192ED03ull));
    r.next();
    return r.next();
}

struct Edge { uint32_t lo, hi; double w; };

// Clique-tree sampling of one eliminated star (Gao-Kyng-Spielman,
// arXiv:2303.00709): neighbours sorted by ascending weight, each one joined to
// a later neighbour drawn in proportion to weight, with weight w_i S_i / d so
// the expected Laplacian equals the exact clique.  `split` copies each
// neighbour edge k times (weight w/k) before sampling, as AC(k) does.
static void sample_star(std::vector<std::pair<uint32_t, double>>& ent, uint32_t split, Rng& rng,
                        std::vector<Edge>& out) {
    if (split > 1) {
        size_t m = ent.size();
        std::vector<std::pair<uint32_t, double>> e2;
        e2.reserve(m * split);
        for (auto& e : ent)
            for (uint32_t s = 0; s < split; ++s) e2.push_back({e.first, e.second / split});
        ent.swap(e2);
    }
    if (ent.size() <= 1) return;
    std::stable_sort(ent.begin(), ent.end(), [](const std::pair<uint32_t, double>& a,
                                                const std::pair<uint32_t, double>& b) {
        if (a.second != b.second) return a.second < b.second;
        return a.first < b.first;
    });
    const size_t m = ent.size();
    std::vector<double> pre(m + 1, 0.0);
    for (size_t i = 0; i < m; ++i) pre[i + 1] = pre[i] + ent[i].second;
    const double d = pre[m];
    for (size_t i = 0; i + 1 < m; ++i) {
        double S = pre[m] - pre[i + 1];
        if (!(S > 0.0)) continue;
        double target = pre[i + 1] + rng.unit() * S;
        size_t j = (size_t)(std::upper_bound(pre.begin() + i + 2, pre.end(), target) - pre.begin()) - 1;
        if (j <= i) j = i + 1;
        if (j >= m) j = m - 1;
        uint32_t a = ent[i].first, b = ent[j].first;
        if (a == b) continue;
        double w = ent[i].second * S / d;
        out.push_back({std::min(a, b), std::max(a, b), w});
    }
}

// Sequential approximate Cholesky of a Laplacian (approx-chol's approximate
// backend, restated from GKS): random elimination order, merged multi-edges,
// clique-tree sampled fill.
static void ac_factor(const SqCsr& m, uint64_t seed, uint32_t split, Factor& f) {
    const size_t n = m.n;
    std::vector<std::vector<std::pair<uint32_t, double>>> adj(n);
    for (size_t i = 0; i < n; ++i)
        for (uint32_t k = m.indptr[i]; k < m.indptr[i + 1]; ++k) {
            uint32_t j = m.indices[k];
            if (j != i && m.data[k] != 0.0) adj[i].push_back({j, -m.data[k]});
        }
    f.n = n;
    f.order.resize(n);
    std::iota(f.order.begin(), f.order.end(), 0u);
    Rng shuffle(mix(seed, 0x5eedull));
    for (size_t i = n; i > 1; --i) std::swap(f.order[i - 1], f.order[shuffle.next() % i]);
    f.pivot.assign(n, 0.0);
    f.colptr.assign(1, 0);
    f.rowidx.clear();
    f.val.clear();
    std::vector<char> gone(n, 0);
    std::vector<double> acc(n, 0.0);
    std::vector<uint32_t> touched;
    std::vector<std::pair<uint32_t, double>> ent;
    std::vector<Edge> fill;
    for (size_t k = 0; k < n; ++k) {
        uint32_t v = f.order[k];
        touched.clear();
        for (auto& e : adj[v]) {
            if (gone[e.first] || e.first == v) continue;
            if (acc[e.first] == 0.0) touched.push_back(e.first);
            acc[e.first] += e.second;
        }
        std::sort(touched.begin(), touched.end());
        ent.clear();
        double d = 0.0;
        for (uint32_t u : touched) {
            if (acc[u] > 0.0) {
                ent.push_back({u, acc[u]});
                d += acc[u];
            }
            acc[u] = 0.0;
        }
        adj[v].clear();
        adj[v].shrink_to_fit();
        gone[v] = 1;
        if (!(d > 0.0)) {
            f.pivot[v] = 0.0;
            f.colptr.push_back((uint32_t)f.rowidx.size());
            continue;
        }
        f.pivot[v] = d;
        for (auto& e : ent) {
            f.rowidx.push_back(e.first);
            f.val.push_back(-e.second / d);
        }
        f.colptr.push_back((uint32_t)f.rowidx.size());
        Rng rng(mix(seed, (uint64_t)v + 1));
        fill.clear();
        sample_star(ent, split, rng, fill);
        for (auto& e : fill) {
            adj[e.lo].push_back({e.hi, e.w});
            adj[e.hi].push_back({e.lo, e.w});
        }
    }
}

// block_elim/factor.rs:157-169 -> approx_chol Builder::build with
// Backend::ExactBelow{max_dim}: dense exact at or below max_dim, else AC.
static bool factor_sparse(const SqCsr& m, uint64_t seed, uint32_t split, size_t max_dim,
                          bool fallback, bool force_dense, Factor& f) {
    if (force_dense || m.n <= max_dim) {
        if (dense_factor(m, f)) return true;
        if (!fallback) return false;
    }
    ac_factor(m, seed, split, f);
    return true;
}

// ---------------------------------------------------------------------------
// SDDM components (domain/factor_pairs/sddm.rs).
enum Grounding { FLOATING = 0, GROUNDED = 1 };

struct Sddm {
    CrossTab ct;
    std::vector<double> diagonal, ground_edges;
    Grounding grounding = FLOATING;
    size_t n_elim() const { return ct.n_rows(); }
    size_t n_kept() const { return ct.n_cols(); }
};

struct Component {
    Sddm m;
    bool laplacian = true;            // MatrixForm::Laplacian vs SignedPendingCover
    std::vector<double> factors;      // empty = CoordinateMap::Canonical
};

static double budget(double ulps, size_t n, double total) {  // sddm.rs:21-25
    return ulps * DBL_EPSILON * std::sqrt((double)std::max<size_t>(n, 1)) * total;
}

static std::vector<double> adjacency_sums(const CrossTab& c, bool magnitude) {
    std::vector<double> s(c.n_local(), 0.0);
    for (size_t i = 0; i < c.n_local(); ++i) {
        double acc = 0.0;
        c.neighbors(i, [&](size_t, double v) { acc += magnitude ? std::fabs(v) : v; });
        s[i] = acc;
    }
    return s;
}

struct Uncert { bool any = false; };

// sddm.rs:172-195
static bool convert_known_laplacian(CrossTab&& ct, std::vector<double>&& diag, Component& out) {
    auto row_sums = adjacency_sums(ct, false);
    double total_diag = 0.0, total_mis = 0.0;
    for (size_t i = 0; i < diag.size(); ++i) {
        total_diag += diag[i];
        total_mis += std::fabs(diag[i] - row_sums[i]);
    }
    if (total_mis > budget(64.0, ct.n_local(), total_diag)) return false;
    out.m.ground_edges.assign(ct.n_local(), 0.0);
    out.m.ct = std::move(ct);
    out.m.diagonal = std::move(row_sums);
    out.m.grounding = FLOATING;
    out.laplacian = true;
    out.factors.clear();
    return true;
}

// sddm.rs:380-407
static bool folding_signs(const CrossTab& ct, std::vector<double>& signs) {
    size_t n = ct.n_local();
    signs.assign(n, 0.0);
    std::vector<size_t> stack;
    for (size_t root = 0; root < n; ++root) {
        if (signs[root] != 0.0) continue;
        signs[root] = 1.0;
        stack.push_back(root);
        bool ok = true;
        while (!stack.empty() && ok) {
            size_t i = stack.back();
            stack.pop_back();
            ct.neighbors(i, [&](size_t j, double v) {
                if (!ok) return;
                double sg = std::signbit(v) ? -1.0 : 1.0;
                double expected = -signs[i] * sg;
                if (signs[j] == 0.0) {
                    signs[j] = expected;
                    stack.push_back(j);
                } else if (signs[j] != expected) {
                    ok = false;
                }
            });
        }
        if (!ok) return false;
    }
    return true;
}

// sddm.rs:416-483
static bool dominance_scaling(const CrossTab& ct, const std::vector<double>& diag,
                              const PrecondCfg& cfg, std::vector<double>& scales, size_t& sweeps,
                              double& violation) {
    size_t n = ct.n_local();
    for (double d : diag)
        if (!std::isfinite(d) || d <= 0.0) return false;
    bool dominant = true;
    for (size_t i = 0; i < n && dominant; ++i) {
        double rs = 0.0;
        ct.neighbors(i, [&](size_t, double v) { rs += std::fabs(v); });
        dominant = rs <= diag[i] * (1.0 + cfg.scaling_tol);
    }
    if (dominant) {
        scales.assign(n, 1.0);
        sweeps = 0;
        violation = 0.0;
        return true;
    }
    std::vector<double> inv_sqrt(n), mu(n, 1.0);
    for (size_t i = 0; i < n; ++i) inv_sqrt[i] = 1.0 / std::sqrt(diag[i]);
    auto target = [&](size_t i) {
        double t = 0.0;
        ct.neighbors(i, [&](size_t j, double v) { t += std::fabs(v) * inv_sqrt[i] * inv_sqrt[j] * mu[j]; });
        return t;
    };
    auto violation_of = [&]() {
        double m = 0.0;
        for (size_t i = 0; i < n; ++i) m = std::fmax(m, target(i) / mu[i] - 1.0);
        return m;
    };
    violation = violation_of();
    sweeps = 0;
    while (violation > cfg.scaling_tol && sweeps < cfg.scaling_max_sweeps) {
        for (size_t i = 0; i < n; ++i) {
            double t = target(i);
            if (t > mu[i]) mu[i] = t;
        }
        double peak = 0.0;
        for (double v : mu) peak = std::fmax(peak, v);
        if (!std::isfinite(peak)) return false;
        for (double& v : mu) v /= peak;
        violation = violation_of();
        sweeps += 1;
    }
    scales.resize(n);
    for (size_t i = 0; i < n; ++i) {
        scales[i] = mu[i] * inv_sqrt[i];
        if (!(std::isfinite(scales[i]) && scales[i] > 0.0)) return false;
    }
    violation = std::max(violation, 0.0);
    return true;
}

// sddm.rs:293-352
static bool finalize(CrossTab&& ct, std::vector<double>&& sd, const std::vector<double>& row_sums,
                     const PrecondCfg& cfg, Component& out, double& clamped) {
    size_t n = ct.n_local();
    std::vector<double> ground(n, 0.0);
    double total_diag = 0.0, total_surplus = 0.0;
    clamped = 0.0;
    for (size_t i = 0; i < n; ++i) {
        double& d = sd[i];
        if (!std::isfinite(d) || d <= 0.0) return false;
        double deficit = (row_sums[i] - d) / d;
        if (deficit > cfg.scaling_tol) {
            if (cfg.scaling_error) return false;
            clamped = std::max(clamped, deficit);
        }
        d = std::max(d, row_sums[i]);
        ground[i] = std::max(d - row_sums[i], 0.0);
        total_diag += d;
        total_surplus += ground[i];
    }
    bool floats = total_surplus <= budget(4.0, n, total_diag);
    if (floats) {
        sd = row_sums;
        std::fill(ground.begin(), ground.end(), 0.0);
    }
    out.m.ct = std::move(ct);
    out.m.diagonal = std::move(sd);
    out.m.ground_edges = std::move(ground);
    out.m.grounding = floats ? FLOATING : GROUNDED;
    return true;
}

// sddm.rs:237-291
static bool assemble(CrossTab&& ct, const std::vector<double>& diag, std::vector<double>&& factors,
                     bool laplacian, const PrecondCfg& cfg, Component& out, double& clamped) {
    size_t nr = ct.n_rows();
    for (size_t i = 0; i < nr; ++i)
        for (uint32_t k = ct.c.indptr[i]; k < ct.c.indptr[i + 1]; ++k) {
            double folded = -factors[i] * factors[nr + ct.c.indices[k]] * ct.c.data[k];
            if (!std::isfinite(folded) || (laplacian && folded < 0.0)) return false;
            ct.c.data[k] = folded;
        }
    ct.ct = transpose(ct.c);
    std::vector<double> sd(diag.size());
    for (size_t i = 0; i < diag.size(); ++i) sd[i] = diag[i] * factors[i] * factors[i];
    bool canonical = true;
    for (size_t i = 0; i < factors.size(); ++i)
        canonical = canonical && factors[i] == (i < nr ? 1.0 : -1.0);
    out.laplacian = laplacian;
    if (canonical)
        out.factors.clear();
    else
        out.factors = std::move(factors);
    auto row_sums = adjacency_sums(ct, true);
    return finalize(std::move(ct), std::move(sd), row_sums, cfg, out, clamped);
}

// sddm.rs:197-235
static bool convert_general(CrossTab&& ct, std::vector<double>&& diag, const PrecondCfg& cfg,
                            Component& out, bool& warn) {
    std::vector<double> signs;
    bool has_signs = folding_signs(ct, signs);
    std::vector<double> scales;
    size_t sweeps = 0;
    double violation = 0.0;
    if (!dominance_scaling(ct, diag, cfg, scales, sweeps, violation)) return false;
    if (violation > cfg.scaling_tol && cfg.scaling_error) return false;
    double clamped = 0.0;
    size_t nr = ct.n_rows();
    if (has_signs) {
        std::vector<double> f(scales.size());
        for (size_t i = 0; i < f.size(); ++i) f[i] = signs[i] * scales[i];
        if (!assemble(std::move(ct), diag, std::move(f), true, cfg, out, clamped)) return false;
    } else {
        for (size_t i = nr; i < scales.size(); ++i) scales[i] = -scales[i];
        if (!assemble(std::move(ct), diag, std::move(scales), false, cfg, out, clamped)) return false;
    }
    warn = std::max(violation, clamped) > cfg.scaling_tol;
    return true;
}

// ---------------------------------------------------------------------------
// Schur complements (block_elim/schur.rs).
static SqCsr exact_principal(const Sddm& m, const std::vector<double>& inv_e) {  // schur.rs:29-62
    size_t nk = m.n_kept();
    SqCsr s;
    s.n = nk;
    std::vector<double> work(nk, 0.0);
    std::vector<size_t> touched;
    const double* dk = &m.diagonal[m.n_elim()];
    for (size_t i = 0; i < nk; ++i) {
        work[i] = dk[i];
        touched.push_back(i);
        for (uint32_t a = m.ct.ct.indptr[i]; a < m.ct.ct.indptr[i + 1]; ++a) {
            uint32_t k = m.ct.ct.indices[a];
            double w = m.ct.ct.data[a];
            double inv = inv_e[k];
            for (uint32_t b = m.ct.c.indptr[k]; b < m.ct.c.indptr[k + 1]; ++b) {
                uint32_t j = m.ct.c.indices[b];
                double v = m.ct.c.data[b];
                if (work[j] == 0.0 && j != i) touched.push_back(j);
                work[j] -= (w * v) * inv;
            }
        }
        std::sort(touched.begin(), touched.end());
        for (size_t j : touched) {
            double v = work[j];
            if (v != 0.0 || j == i) {
                s.indices.push_back((uint32_t)j);
                s.data.push_back(v);
            }
            work[j] = 0.0;
        }
        touched.clear();
        s.indptr.push_back((uint32_t)s.indices.size());
    }
    return s;
}

static std::vector<double> reduced_surplus(const Sddm& m, const std::vector<double>& inv_e) {
    std::vector<double> out(m.n_kept(), 0.0);
    if (m.grounding == FLOATING) return out;
    std::vector<double> scaled(m.n_elim());
    for (size_t k = 0; k < m.n_elim(); ++k) scaled[k] = inv_e[k] * m.ground_edges[k];
    spmv_assign_add(m.ct.ct, scaled.data(), &m.ground_edges[m.n_elim()], out.data());
    return out;
}

// schur.rs:228-272
static SqCsr build_explicit_laplacian(const SqCsr& p, const std::vector<double>& surplus,
                                      Grounding g) {
    size_t nk = p.n;
    bool grounded = g == GROUNDED;
    SqCsr out;
    out.n = nk + (grounded ? 1 : 0);
    for (size_t i = 0; i < nk; ++i) {
        double adjacency = 0.0;
        long dpos = -1;
        for (uint32_t k = p.indptr[i]; k < p.indptr[i + 1]; ++k) {
            uint32_t j = p.indices[k];
            if (j == i) {
                dpos = (long)out.indices.size();
                out.indices.push_back(j);
                out.data.push_back(0.0);
            } else {
                adjacency -= p.data[k];
                out.indices.push_back(j);
                out.data.push_back(p.data[k]);
            }
        }
        out.data[dpos] = adjacency + surplus[i];
        if (grounded && surplus[i] > 0.0) {
            out.indices.push_back((uint32_t)nk);
            out.data.push_back(-surplus[i]);
        }
        out.indptr.push_back((uint32_t)out.indices.size());
    }
    if (grounded) {
        for (size_t i = 0; i < nk; ++i)
            if (surplus[i] > 0.0) {
                out.indices.push_back((uint32_t)i);
                out.data.push_back(-surplus[i]);
            }
        out.indices.push_back((uint32_t)nk);
        out.data.push_back(compensated_sum(surplus.data(), surplus.size()));
        out.indptr.push_back((uint32_t)out.indices.size());
    }
    return out;
}

static SqCsr exact_for_factor(const Sddm& m, const std::vector<double>& inv_e) {
    return build_explicit_laplacian(exact_principal(m, inv_e), reduced_surplus(m, inv_e), m.grounding);
}

// schur.rs:64-68, 116-226, 337-429 -- sampled Schur on the explicit augmented graph.
static SqCsr laplacian_from_edges(std::vector<Edge>& edges, size_t n) {
    std::sort(edges.begin(), edges.end(), [](const Edge& a, const Edge& b) {
        if (a.lo != b.lo) return a.lo < b.lo;
        if (a.hi != b.hi) return a.hi < b.hi;
        return a.w < b.w;
    });
    std::vector<Edge> dd;
    for (auto& e : edges) {
        if (!dd.empty() && dd.back().lo == e.lo && dd.back().hi == e.hi)
            dd.back().w += e.w;
        else
            dd.push_back(e);
    }
    std::vector<uint32_t> lower(n, 0), upper(n, 0);
    std::vector<double> diag(n, 0.0);
    for (auto& e : dd) {
        diag[e.lo] += e.w;
        upper[e.lo] += 1;
        lower[e.hi] += 1;
        diag[e.hi] += e.w;
    }
    SqCsr s;
    s.n = n;
    s.indptr.assign(n + 1, 0);
    for (size_t i = 0; i < n; ++i) s.indptr[i + 1] = s.indptr[i] + lower[i] + 1 + upper[i];
    s.indices.assign(s.indptr[n], 0);
    s.data.assign(s.indptr[n], 0.0);
    std::vector<uint32_t> lc(n), uc(n);
    for (size_t i = 0; i < n; ++i) {
        lc[i] = s.indptr[i];
        uc[i] = s.indptr[i] + lower[i] + 1;
        uint32_t pos = s.indptr[i] + lower[i];
        s.indices[pos] = (uint32_t)i;
        s.data[pos] = diag[i];
    }
    for (auto& e : dd) {
        uint32_t p = uc[e.lo]++;
        s.indices[p] = e.hi;
        s.data[p] = -e.w;
        p = lc[e.hi]++;
        s.indices[p] = e.lo;
        s.data[p] = -e.w;
    }
    return s;
}

static SqCsr sampled_schur(const Sddm& m, uint64_t seed, uint32_t split) {
    size_t nk = m.n_kept();
    bool grounded = m.grounding == GROUNDED;
    std::vector<Edge> edges;
    std::vector<std::pair<uint32_t, double>> ent;
    for (size_t k = 0; k < m.n_elim(); ++k) {
        ent.clear();
        for (uint32_t a = m.ct.c.indptr[k]; a < m.ct.c.indptr[k + 1]; ++a)
            ent.push_back({m.ct.c.indices[a], m.ct.c.data[a]});
        if (ent.empty()) continue;
        if (grounded && m.ground_edges[k] > 0.0) ent.push_back({(uint32_t)nk, m.ground_edges[k]});
        if (ent.size() <= 1) continue;
        Rng rng(mix(seed, (uint64_t)k));
        sample_star(ent, split, rng, edges);
    }
    if (grounded)
        for (size_t i = 0; i < nk; ++i)
            if (m.ground_edges[m.n_elim() + i] > 0.0)
                edges.push_back({(uint32_t)i, (uint32_t)nk, m.ground_edges[m.n_elim() + i]});
    return laplacian_from_edges(edges, nk + (grounded ? 1 : 0));
}

// ---------------------------------------------------------------------------
// Block-elimination local solver (block_elim/solver.rs).
struct BlockElim {
    CrossTab ct;
    std::vector<double> inv_e;
    Factor factor;
    bool cover = false;
    Grounding grounding = FLOATING;   // Direct factor's gauge
    size_t n_internal = 0, n_reduced = 0;
    std::vector<double> factors;      // empty = Canonical

    size_t n_elim() const { return ct.n_rows(); }
    size_t n_kept() const { return ct.n_cols(); }
    bool explicit_ground() const { return !cover && grounding == GROUNDED && factor.n == n_kept() + 1; }

    void fold(double* v) const {  // sddm.rs:61-83
        if (factors.empty()) {
            for (size_t i = n_elim(); i < n_internal; ++i) v[i] = -v[i];
        } else {
            for (size_t i = 0; i < n_internal; ++i) v[i] *= factors[i];
        }
    }
    static void subtract_mean(double* s, size_t n) {  // solver.rs:21-31
        if (n == 0) return;
        double mean = compensated_sum(s, n) / (double)n;
        for (size_t i = 0; i < n; ++i) s[i] -= mean;
    }
    void reduced_solve(double* x, std::vector<double>& scratch) const {  // factor.rs:78-110
        if (!cover) {
            factor.solve_in_place(x);
            return;
        }
        size_t m = n_kept(), cn = factor.n;
        scratch.assign(cn, 0.0);
        for (size_t i = 0; i < m; ++i) {
            scratch[i] = x[i];
            scratch[m + i] = -x[i];
        }
        factor.solve_in_place(scratch.data());
        for (size_t i = 0; i < m; ++i) x[i] = 0.5 * (scratch[i] - scratch[m + i]);
    }
    // solver.rs:445-466 and eliminate_and_recover 350-423
    void solve_local(std::vector<double>& rhs, std::vector<double>& sol) const {
        const size_t n = n_internal, ne = n_elim(), nk = n_kept();
        fold(rhs.data());
        bool floating = !cover && grounding == FLOATING;
        if (floating) subtract_mean(rhs.data(), n);
        for (size_t i = 0; i < ne; ++i) rhs[i] *= inv_e[i];
        std::vector<double> red(n_reduced, 0.0);
        spmv_assign_add(ct.ct, rhs.data(), rhs.data() + ne, red.data());
        if (floating) {
            subtract_mean(red.data(), n_reduced);
        } else if (explicit_ground()) {
            red[nk] = -compensated_sum(red.data(), nk);
        }
        std::vector<double> scratch;
        reduced_solve(red.data(), scratch);
        if (explicit_ground()) {
            double g = red[nk];
            for (size_t i = 0; i < nk; ++i) red[i] -= g;
        }
        sol.assign(n, 0.0);
        for (size_t i = 0; i < nk; ++i) sol[ne + i] = red[i];
        for (size_t i = 0; i < ne; ++i) {
            double s = 0.0;
            for (uint32_t k = ct.c.indptr[i]; k < ct.c.indptr[i + 1]; ++k)
                s += ct.c.data[k] * red[ct.c.indices[k]];
            sol[i] = rhs[i] + inv_e[i] * s;
        }
        if (floating) subtract_mean(sol.data(), n);
        fold(sol.data());
    }
};

// Gremban cover of a signed matrix (solver.rs:220-271).
static Sddm bipartite_cover(const Sddm& m) {
    const Csr& c = m.ct.c;
    size_t nr = c.nrows, nc = c.ncols;
    Csr cc;
    cc.nrows = 2 * nr;
    cc.ncols = 2 * nc;
    for (int copy = 0; copy < 2; ++copy)
        for (size_t i = 0; i < nr; ++i) {
            for (int cs = 0; cs < 2; ++cs) {
                uint32_t base = cs ? (uint32_t)nc : 0u;
                bool sel_neg = (cs != 0) != (copy != 0);
                for (uint32_t k = c.indptr[i]; k < c.indptr[i + 1]; ++k) {
                    double v = c.data[k];
                    if ((v < 0.0) != sel_neg) continue;
                    cc.indices.push_back(c.indices[k] + base);
                    cc.data.push_back(std::fabs(v));
                }
            }
            cc.indptr.push_back((uint32_t)cc.indices.size());
        }
    auto dbl = [&](const std::vector<double>& v) {
        std::vector<double> o;
        o.insert(o.end(), v.begin(), v.begin() + nr);
        o.insert(o.end(), v.begin(), v.begin() + nr);
        o.insert(o.end(), v.begin() + nr, v.end());
        o.insert(o.end(), v.begin() + nr, v.end());
        return o;
    };
    Sddm out;
    out.ct.c = cc;
    out.ct.ct = transpose(cc);
    out.diagonal = dbl(m.diagonal);
    out.ground_edges = dbl(m.ground_edges);
    out.grounding = m.grounding;
    return out;
}

static std::vector<double> inv_elim(const Sddm& m) {
    std::vector<double> inv(m.n_elim());
    for (size_t i = 0; i < m.n_elim(); ++i) {
        double d = m.diagonal[i];
        if (!(d > 0.0)) throw Error(E_SINGULAR, "zero diagonal in preconditioner at index " + std::to_string(i));
        inv[i] = 1.0 / d;
    }
    return inv;
}

// solver.rs:191-217 -- factor_reduced
static void factor_reduced(const Sddm& m, const std::vector<double>& inv_e, const PrecondCfg& cfg,
                           Factor& f) {
    size_t eb = cfg.dense_threshold;
    if (cfg.exact_local) {
        SqCsr ex = exact_for_factor(m, inv_e);
        factor_sparse(ex, cfg.ac_seed, cfg.ac_split, eb, true, true, f);
        return;
    }
    bool have_exact = eb > 0 && m.n_kept() <= eb;
    SqCsr ex;
    if (have_exact) {
        ex = exact_for_factor(m, inv_e);
        if (factor_sparse(ex, cfg.ac_seed, cfg.ac_split, eb, false, false, f)) return;
    }
    SqCsr comp = cfg.schur_exact ? (have_exact ? ex : exact_for_factor(m, inv_e))
                                 : sampled_schur(m, cfg.schur_seed, cfg.schur_split);
    factor_sparse(comp, cfg.ac_seed, cfg.ac_split, eb, true, false, f);
}

static BlockElim build_block_elim(Component&& comp, const PrecondCfg& cfg) {
    BlockElim s;
    std::vector<double> inv_e = inv_elim(comp.m);
    if (comp.laplacian) {
        factor_reduced(comp.m, inv_e, cfg, s.factor);
        s.cover = false;
        s.grounding = comp.m.grounding;
        s.n_reduced = s.factor.n;
    } else {
        Sddm cov = bipartite_cover(comp.m);
        std::vector<double> inv_c = inv_elim(cov);
        factor_reduced(cov, inv_c, cfg, s.factor);
        s.cover = true;
        s.n_reduced = comp.m.n_kept();
    }
    s.ct = std::move(comp.m.ct);
    s.inv_e = std::move(inv_e);
    s.factors = std::move(comp.factors);
    s.n_internal = s.ct.n_local();
    return s;
}

// ---------------------------------------------------------------------------
// Additive Schwarz (schwarz-precond/src/{domain,local_solve}.rs, executor.rs).
struct Subdomain {
    std::vector<uint32_t> globals;
    std::vector<double> pw;  // empty = uniform
    BlockElim solver;
};

struct SchwarzPrecond : Preconditioner {
    std::vector<Subdomain> subs;
    size_t n_subdomains() const override { return subs.size(); }
    void apply(const double* r, double* z) const override {
        for (size_t i = 0; i < n; ++i) z[i] = 0.0;
        if (g_threads > 1 && subs.size() > 1) {
            // timing mode: subdomains concurrently (executor.rs:55-166), each
            // into its own buffer, added in subdomain order
            std::vector<std::vector<double>> zs(subs.size());
            std::vector<std::thread> pool;
            for (size_t q = 0; q < subs.size(); ++q)
                pool.emplace_back([&, q] {
                    const auto& s = subs[q];
                    const size_t nl = s.globals.size();
                    std::vector<double> rl(nl, 0.0), sl;
                    for (size_t i = 0; i < nl; ++i)
                        rl[i] = s.pw.empty() ? r[s.globals[i]] : r[s.globals[i]] * s.pw[i];
                    s.solver.solve_local(rl, sl);
                    zs[q].resize(nl);
                    for (size_t i = 0; i < nl; ++i) zs[q][i] = s.pw.empty() ? sl[i] : sl[i] * s.pw[i];
                });
            for (auto& th : pool) th.join();
            for (size_t q = 0; q < subs.size(); ++q)
                for (size_t i = 0; i < subs[q].globals.size(); ++i) z[subs[q].globals[i]] += zs[q][i];
            return;
        }
        std::vector<double> rl, sl;
        for (const auto& s : subs) {
            size_t nl = s.globals.size();
            rl.assign(nl, 0.0);
            for (size_t i = 0; i < nl; ++i)
                rl[i] = s.pw.empty() ? r[s.globals[i]] : r[s.globals[i]] * s.pw[i];
            s.solver.solve_local(rl, sl);
            for (size_t i = 0; i < nl; ++i)
                z[s.globals[i]] += s.pw.empty() ? sl[i] : sl[i] * s.pw[i];
        }
    }
};

// factor_pairs.rs:36-194 with cross_tab.rs and accumulate.rs.
static SchwarzPrecond* build_additive(const Design& d, const double* weights, const PrecondCfg& cfg,
                                      size_t& n_warn) {
    struct Ch { size_t term, column; };
    std::vector<Ch> channels;
    for (size_t t = 0; t < d.terms.size(); ++t)
        for (size_t c = 0; c < d.terms[t].n_columns(); ++c) channels.push_back({t, c});
    std::vector<std::vector<char>> active(d.terms.size());
    for (size_t t = 0; t < d.terms.size(); ++t) {
        active[t].assign(d.terms[t].n_levels, 0);
        for (uint32_t v : d.codes[t]) active[t][v] = 1;
    }
    bool any_slope = false;
    for (auto& ch : channels) any_slope = any_slope || d.terms[ch.term].columns[ch.column] >= 0;

    auto* P = new SchwarzPrecond();
    P->n = d.n_dofs;
    for (size_t a = 0; a < channels.size(); ++a)
        for (size_t b = a + 1; b < channels.size(); ++b) {
            Ch R = channels[a], C = channels[b];
            if (R.term == C.term) continue;
            // build_compact_mapping (cross_tab.rs:46-82)
            const auto& ar = active[R.term];
            const auto& ac = active[C.term];
            std::vector<uint32_t> rmap(ar.size(), UINT32_MAX), cmap(ac.size(), UINT32_MAX), l2g;
            size_t nr = 0, nc = 0;
            size_t base_r = d.terms[R.term].column_base(R.column);
            size_t base_c = d.terms[C.term].column_base(C.column);
            for (size_t j = 0; j < ar.size(); ++j)
                if (ar[j]) { rmap[j] = (uint32_t)nr++; l2g.push_back((uint32_t)(base_r + j)); }
            for (size_t k = 0; k < ac.size(); ++k)
                if (ac[k]) { cmap[k] = (uint32_t)nc++; l2g.push_back((uint32_t)(base_c + k)); }
            if (nr == 0 || nc == 0) continue;
            // accumulate (accumulate.rs:86-273): both routes sum each cell in
            // observation order, so the sparse route is used unconditionally.
            const uint32_t* rl = d.codes[R.term].data();
            const uint32_t* cl = d.codes[C.term].data();
            int kr = d.terms[R.term].columns[R.column], kc = d.terms[C.term].columns[C.column];
            std::vector<double> rdiag(nr, 0.0), cdiag(nc, 0.0);
            std::vector<uint32_t> cnt(nr + 1, 0);
            for (size_t i = 0; i < d.n_obs; ++i) cnt[rmap[rl[i]] + 1] += 1;
            for (size_t i = 0; i < nr; ++i) cnt[i + 1] += cnt[i];
            std::vector<uint32_t> bcol(d.n_obs), cur(cnt.begin(), cnt.end() - 1);
            std::vector<double> bval(d.n_obs);
            for (size_t i = 0; i < d.n_obs; ++i) {
                uint32_t cj = rmap[rl[i]], ck = cmap[cl[i]];
                double w = weights ? weights[i] : 1.0;
                double lr = kr < 0 ? 1.0 : d.loads[kr][i];
                double lc = kc < 0 ? 1.0 : d.loads[kc][i];
                rdiag[cj] += w * lr * lr;
                cdiag[ck] += w * lc * lc;
                uint32_t p = cur[cj]++;
                bcol[p] = ck;
                bval[p] = w * lr * lc;
            }
            CrossTab full;
            full.c.nrows = nr;
            full.c.ncols = nc;
            std::vector<double> work(nc, 0.0);
            std::vector<uint32_t> touched;
            for (size_t r = 0; r < nr; ++r) {
                for (uint32_t p = cnt[r]; p < cnt[r + 1]; ++p) {
                    uint32_t col = bcol[p];
                    if (work[col] == 0.0) touched.push_back(col);
                    work[col] += bval[p];
                }
                std::sort(touched.begin(), touched.end());
                touched.erase(std::unique(touched.begin(), touched.end()), touched.end());
                for (uint32_t col : touched) {
                    if (work[col] != 0.0) {
                        full.c.indices.push_back(col);
                        full.c.data.push_back(work[col]);
                    }
                    work[col] = 0.0;
                }
                full.c.indptr.push_back((uint32_t)full.c.indices.size());
                touched.clear();
            }
            full.ct = transpose(full.c);
            bool known_lap = kr < 0 && kc < 0;
            // bipartite_connected_components (cross_tab.rs:175-211)
            size_t nl = nr + nc;
            std::vector<char> vis(nl, 0);
            std::vector<size_t> stack;
            std::vector<std::pair<std::vector<size_t>, std::vector<size_t>>> comps;
            for (size_t s = 0; s < nl; ++s) {
                if (vis[s]) continue;
                vis[s] = 1;
                stack.push_back(s);
                std::vector<size_t> rows, cols;
                while (!stack.empty()) {
                    size_t node = stack.back();
                    stack.pop_back();
                    if (node < nr) rows.push_back(node); else cols.push_back(node - nr);
                    full.neighbors(node, [&](size_t j, double) {
                        if (!vis[j]) { vis[j] = 1; stack.push_back(j); }
                    });
                }
                std::sort(rows.begin(), rows.end());
                std::sort(cols.begin(), cols.end());
                comps.push_back({rows, cols});
            }
            std::vector<uint32_t> rremap(nr, UINT32_MAX), cremap(nc, UINT32_MAX);
            for (auto& comp : comps) {
                CrossTab ct;
                std::vector<double> diag;
                if (comps.size() == 1) {
                    ct = full;
                    diag = rdiag;
                    diag.insert(diag.end(), cdiag.begin(), cdiag.end());
                } else {  // extract_component (cross_tab.rs:214-268)
                    for (size_t i = 0; i < comp.first.size(); ++i) rremap[comp.first[i]] = (uint32_t)i;
                    for (size_t i = 0; i < comp.second.size(); ++i) cremap[comp.second[i]] = (uint32_t)i;
                    ct.c.nrows = comp.first.size();
                    ct.c.ncols = comp.second.size();
                    for (size_t orow : comp.first) {
                        for (uint32_t k = full.c.indptr[orow]; k < full.c.indptr[orow + 1]; ++k) {
                            uint32_t nj = cremap[full.c.indices[k]];
                            if (nj != UINT32_MAX) { ct.c.indices.push_back(nj); ct.c.data.push_back(full.c.data[k]); }
                        }
                        ct.c.indptr.push_back((uint32_t)ct.c.indices.size());
                    }
                    ct.ct = transpose(ct.c);
                    for (size_t o : comp.first) rremap[o] = UINT32_MAX;
                    for (size_t o : comp.second) cremap[o] = UINT32_MAX;
                    for (size_t o : comp.first) diag.push_back(rdiag[o]);
                    for (size_t o : comp.second) diag.push_back(cdiag[o]);
                }
                bool allzero = true;
                for (double v : diag) allzero = allzero && v == 0.0;
                if (allzero) continue;
                std::vector<uint32_t> globals;
                for (size_t o : comp.first) globals.push_back(l2g[o]);
                for (size_t o : comp.second) globals.push_back(l2g[nr + o]);
                // orient_for_elimination (sddm.rs:85-106)
                if (ct.n_cols() > ct.n_rows()) {
                    size_t k = ct.n_rows();
                    std::rotate(diag.begin(), diag.begin() + k, diag.end());
                    std::rotate(globals.begin(), globals.begin() + k, globals.end());
                    std::swap(ct.c, ct.ct);
                }
                Component cp;
                bool warn = false, ok;
                if (known_lap)
                    ok = convert_known_laplacian(std::move(ct), std::move(diag), cp);
                else
                    ok = convert_general(std::move(ct), std::move(diag), cfg, cp, warn);
                if (!ok) {
                    delete P;
                    throw Error(E_SCALING, "signed component is not diagonally scalable to SDDM form");
                }
                if (warn) n_warn += 1;
                Subdomain sd;
                sd.globals = std::move(globals);
                sd.solver = build_block_elim(std::move(cp), cfg);
                P->subs.push_back(std::move(sd));
            }
        }
    if (!any_slope) {  // compute_partition_weights (factor_pairs.rs:154-194)
        std::vector<uint32_t> counts(d.n_dofs, 0);
        for (auto& s : P->subs)
            for (uint32_t g : s.globals) counts[g] += 1;
        for (auto& s : P->subs) {
            bool uniq = true;
            for (uint32_t g : s.globals) uniq = uniq && counts[g] <= 1;
            if (uniq) continue;
            s.pw.resize(s.globals.size());
            for (size_t i = 0; i < s.globals.size(); ++i) s.pw[i] = 1.0 / std::sqrt((double)counts[s.globals[i]]);
        }
    }
    return P;
}

// operator/schwarz.rs:231-270
BuildOut build_preconditioner(const Design& d, const double* weights, const PrecondCfg& cfg) {
    BuildOut out;
    if (cfg.kind == 0) return out;
    if (cfg.kind == 2) {
        out.precond = build_diagonal(d, weights);
        return out;
    }
    size_t nw = 0;
    SchwarzPrecond* p = build_additive(d, weights, cfg, nw);
    out.n_warnings = nw;
    if (p->subs.empty()) {
        delete p;
        return out;
    }
    out.precond = p;
    return out;
}

}  // namespace orc
