// host_schwarz.cpp -- construction of the Diagonal and additive-Schwarz
// preconditioners (once per Solver, host side), packed for the GPU apply.
//
// Construction follows the reference's steps (crates/within/src/domain/
// {cross_tab,factor_pairs}*, block_elim/*, operator/schwarz.rs):
//   channel pairs -> weighted cross-tab C of active levels -> bipartite
//   connected components -> orient (eliminate the larger block) -> SDDM form
//   (known Laplacian, or signed/scaled General with a Gremban cover when
//   frustrated) -> partition-of-unity weights -> reduced system
//   D_k - C^T D_e^-1 C (exact for small kept blocks, clique-tree sampled
//   otherwise) as an explicit Laplacian.
// The reduced Laplacian is then factored for the GPU:
//   * n <= DENSE_MAX: dense LDL^T with a pseudo-inverse pivot, stored as the
//     dense generalised inverse (one batched mat-vec per apply).  For the
//     reference's exact route (n_kept <= dense_threshold) this is the same
//     operator the reference applies.
//   * otherwise: approximate Cholesky (Gao-Kyng-Spielman clique-tree sampling,
//     arXiv:2303.00709) whose elimination proceeds in rounds of independent
//     vertices.  Vertices of one round share no edge, so their columns are
//     computed from the same graph and the triangular solves run one round
//     per parallel step (level scheduling by construction).
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cfloat>
#include <cmath>
#include <exception>
#include <functional>
#include <numeric>
#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <mutex>
#include <thread>
#include <type_traits>

#include "host.hpp"
#include "host_pool.hpp"

namespace wgpu {
namespace {

// WITHIN_TRACE=1: phase times of the build, one line each on stderr (a
// diagnostic; no effect on results)
struct BuildTrace {
    const char* what;
    long idx;
    double t0;
    static bool on() {
        static const bool v = [] {
            const char* e = std::getenv("WITHIN_TRACE");
            return e && std::atoi(e) != 0;
        }();
        return v;
    }
    static double now() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
    }
    explicit BuildTrace(const char* w, long i = -1) : what(w), idx(i), t0(on() ? now() : 0.0) {}
    void done() {
        if (!on() || !what) return;
        if (idx >= 0) fprintf(stderr, "[within trace]   %s %ld %.3f ms\n", what, idx, (now() - t0) * 1e3);
        else fprintf(stderr, "[within trace]   %s %.3f ms\n", what, (now() - t0) * 1e3);
        what = nullptr;
    }
    ~BuildTrace() { done(); }
};

// WITHIN_TRACE=1: time spent in the named steps of a loop, summed over its
// passes and printed as one line when the loop's owner goes out of scope
struct StepTimes {
    const char* what;
    const char* const* names;
    int n;
    double t[8] = {};
    double last = 0.0;
    StepTimes(const char* w, const char* const* nm, int k) : what(w), names(nm), n(k) {
        if (BuildTrace::on()) last = BuildTrace::now();
    }
    void mark(int i) {
        if (!BuildTrace::on()) return;
        const double x = BuildTrace::now();
        t[i] += x - last;
        last = x;
    }
    ~StepTimes() {
        if (!BuildTrace::on()) return;
        fprintf(stderr, "[within trace]       %s:", what);
        for (int i = 0; i < n; ++i) fprintf(stderr, " %s %.3f ms", names[i], t[i] * 1e3);
        fprintf(stderr, "\n");
    }
};

constexpr uint32_t DENSE_MAX = 64;

struct Csr {
    std::vector<uint32_t> ptr{0}, col;
    std::vector<double> val;
    uint32_t nr = 0, nc = 0;
    uint32_t nnz() const { return (uint32_t)val.size(); }
};

Csr transpose(const Csr& a) {
    Csr t;
    t.nr = a.nc;
    t.nc = a.nr;
    if (a.nnz() >= (1u << 18) && a.nr >= 64) {
        // chunks of rows count their entries per column and scatter side by
        // side; every column receives its entries in ascending row order
        const size_t nch = 16;
        std::vector<uint32_t> rb(nch + 1, a.nr);   // chunk t = rows [rb[t], rb[t+1])
        {
            const uint64_t goal = ((uint64_t)a.nnz() + nch - 1) / nch;
            size_t t = 1;
            rb[0] = 0;
            for (uint32_t r = 0; r < a.nr && t < nch; ++r)
                if ((uint64_t)a.ptr[r + 1] >= goal * t) rb[t++] = r + 1;
        }
        std::vector<std::vector<uint32_t>> cnt(nch);
        par_for_each(nch, [&](size_t c) {
            cnt[c].assign(a.nc, 0);
            for (uint32_t k = a.ptr[rb[c]]; k < a.ptr[rb[c + 1]]; ++k) ++cnt[c][a.col[k]];
        });
        t.ptr.assign(a.nc + 1, 0);
        for (uint32_t j = 0; j < a.nc; ++j) {
            uint32_t o = t.ptr[j];
            for (size_t c = 0; c < nch; ++c) {
                const uint32_t n = cnt[c][j];
                cnt[c][j] = o;
                o += n;
            }
            t.ptr[j + 1] = o;
        }
        t.col.resize(a.nnz());
        t.val.resize(a.nnz());
        par_for_each(nch, [&](size_t c) {
            std::vector<uint32_t>& cur = cnt[c];
            for (uint32_t r = rb[c]; r < rb[c + 1]; ++r)
                for (uint32_t k = a.ptr[r]; k < a.ptr[r + 1]; ++k) {
                    const uint32_t p = cur[a.col[k]]++;
                    t.col[p] = r;
                    t.val[p] = a.val[k];
                }
        });
        return t;
    }
    t.ptr.assign(a.nc + 1, 0);
    for (uint32_t c : a.col) ++t.ptr[c + 1];
    for (uint32_t i = 0; i < a.nc; ++i) t.ptr[i + 1] += t.ptr[i];
    std::vector<uint32_t> cur(t.ptr.begin(), t.ptr.end() - 1);
    t.col.resize(a.nnz());
    t.val.resize(a.nnz());
    for (uint32_t r = 0; r < a.nr; ++r)
        for (uint32_t k = a.ptr[r]; k < a.ptr[r + 1]; ++k) {
            uint32_t p = cur[a.col[k]]++;
            t.col[p] = r;
            t.val[p] = a.val[k];
        }
    return t;
}

struct Bip {  // C (rows = first block) and C^T
    Csr c, ct;
    uint32_t nr() const { return c.nr; }
    uint32_t nc() const { return c.nc; }
    uint32_t nl() const { return c.nr + c.nc; }
    template <class F>
    void nb(uint32_t i, F f) const {
        if (i < c.nr) {
            for (uint32_t k = c.ptr[i]; k < c.ptr[i + 1]; ++k) f(c.nr + c.col[k], c.val[k]);
        } else {
            uint32_t r = i - c.nr;
            for (uint32_t k = ct.ptr[r]; k < ct.ptr[r + 1]; ++k) f(ct.col[k], ct.val[k]);
        }
    }
};

double neumaier(const double* v, size_t n) {
    double s = 0, c = 0;
    for (size_t i = 0; i < n; ++i) {
        double t = s + v[i];
        c += std::fabs(s) >= std::fabs(v[i]) ? (s - t) + v[i] : (v[i] - t) + s;
        s = t;
    }
    return s + c;
}

// ---- SDDM conversion (domain/factor_pairs/sddm.rs) ----
struct Comp {
    Bip m;
    std::vector<double> diag, ground;
    bool grounded = false;
    bool laplacian = true;      // false: signed, needs the Gremban cover
    std::vector<double> factors;  // empty: canonical (negate kept block)
};

double budget(double ulps, size_t n, double total) {
    return ulps * DBL_EPSILON * std::sqrt((double)std::max<size_t>(n, 1)) * total;
}

std::vector<double> sums(const Bip& m, bool mag) {
    std::vector<double> s(m.nl());
    auto range = [&](uint32_t i0, uint32_t i1) {
        for (uint32_t i = i0; i < i1; ++i) {
            double a = 0;
            m.nb(i, [&](uint32_t, double v) { a += mag ? std::fabs(v) : v; });
            s[i] = a;
        }
    };
    const uint32_t B = 16384;
    if (m.c.nnz() >= (1u << 18))
        par_for_each(((size_t)m.nl() + B - 1) / B, [&](size_t b) {
            range((uint32_t)(b * B), (uint32_t)std::min<size_t>(m.nl(), (b + 1) * (size_t)B));
        });
    else range(0, m.nl());
    return s;
}

bool finalize(Comp& c, std::vector<double> sd, const std::vector<double>& rs, const PrecondCfg& cfg,
              double& clamped) {
    size_t n = sd.size();
    std::vector<double> g(n, 0.0);
    double td = 0, ts = 0;
    clamped = 0;
    for (size_t i = 0; i < n; ++i) {
        double& d = sd[i];
        if (!std::isfinite(d) || d <= 0.0) return false;
        double deficit = (rs[i] - d) / d;
        if (deficit > cfg.scaling_tol) {
            if (cfg.scaling_error) return false;
            clamped = std::max(clamped, deficit);
        }
        d = std::max(d, rs[i]);
        g[i] = std::max(d - rs[i], 0.0);
        td += d;
        ts += g[i];
    }
    bool floats = ts <= budget(4.0, n, td);
    if (floats) {
        sd = rs;
        std::fill(g.begin(), g.end(), 0.0);
    }
    c.diag = std::move(sd);
    c.ground = std::move(g);
    c.grounded = !floats;
    return true;
}

bool convert_general(Comp& c, const std::vector<double>& diag, const PrecondCfg& cfg, bool& warn) {
    const uint32_t n = c.m.nl(), nr = c.m.nr();
    // folding signs: a bipartite signature making every off-diagonal <= 0
    std::vector<double> sg(n, 0.0);
    bool has_sg = true;
    std::vector<uint32_t> st;
    for (uint32_t r = 0; r < n && has_sg; ++r) {
        if (sg[r] != 0.0) continue;
        sg[r] = 1.0;
        st.push_back(r);
        while (!st.empty() && has_sg) {
            uint32_t i = st.back();
            st.pop_back();
            c.m.nb(i, [&](uint32_t j, double v) {
                double e = -sg[i] * (std::signbit(v) ? -1.0 : 1.0);
                if (sg[j] == 0.0) {
                    sg[j] = e;
                    st.push_back(j);
                } else if (sg[j] != e) {
                    has_sg = false;
                }
            });
        }
    }
    // dominance scaling (sddm.rs:416-483)
    for (double d : diag)
        if (!std::isfinite(d) || d <= 0.0) return false;
    std::vector<double> scales(n, 1.0);
    double violation = 0.0;
    bool dom = true;
    for (uint32_t i = 0; i < n && dom; ++i) {
        double rs = 0;
        c.m.nb(i, [&](uint32_t, double v) { rs += std::fabs(v); });
        dom = rs <= diag[i] * (1.0 + cfg.scaling_tol);
    }
    if (!dom) {
        std::vector<double> is(n), mu(n, 1.0);
        for (uint32_t i = 0; i < n; ++i) is[i] = 1.0 / std::sqrt(diag[i]);
        auto target = [&](uint32_t i) {
            double t = 0;
            c.m.nb(i, [&](uint32_t j, double v) { t += std::fabs(v) * is[i] * is[j] * mu[j]; });
            return t;
        };
        auto viol = [&]() {
            double m = 0;
            for (uint32_t i = 0; i < n; ++i) m = std::fmax(m, target(i) / mu[i] - 1.0);
            return m;
        };
        violation = viol();
        uint64_t sweeps = 0;
        while (violation > cfg.scaling_tol && sweeps < cfg.scaling_max_sweeps) {
            for (uint32_t i = 0; i < n; ++i) {
                double t = target(i);
                if (t > mu[i]) mu[i] = t;
            }
            double pk = 0;
            for (double v : mu) pk = std::fmax(pk, v);
            if (!std::isfinite(pk)) return false;
            for (double& v : mu) v /= pk;
            violation = viol();
            ++sweeps;
        }
        for (uint32_t i = 0; i < n; ++i) {
            scales[i] = mu[i] * is[i];
            if (!(std::isfinite(scales[i]) && scales[i] > 0.0)) return false;
        }
        violation = std::max(violation, 0.0);
    }
    if (violation > cfg.scaling_tol && cfg.scaling_error) return false;
    std::vector<double> f(n);
    if (has_sg) {
        for (uint32_t i = 0; i < n; ++i) f[i] = sg[i] * scales[i];
    } else {
        for (uint32_t i = 0; i < n; ++i) f[i] = i < nr ? scales[i] : -scales[i];
    }
    // assemble (sddm.rs:237-291)
    for (uint32_t i = 0; i < nr; ++i)
        for (uint32_t k = c.m.c.ptr[i]; k < c.m.c.ptr[i + 1]; ++k) {
            double fo = -f[i] * f[nr + c.m.c.col[k]] * c.m.c.val[k];
            if (!std::isfinite(fo) || (has_sg && fo < 0.0)) return false;
            c.m.c.val[k] = fo;
        }
    c.m.ct = transpose(c.m.c);
    std::vector<double> sd(n);
    for (uint32_t i = 0; i < n; ++i) sd[i] = diag[i] * f[i] * f[i];
    bool canonical = true;
    for (uint32_t i = 0; i < n; ++i) canonical = canonical && f[i] == (i < nr ? 1.0 : -1.0);
    c.laplacian = has_sg;
    c.factors = canonical ? std::vector<double>() : f;
    double clamped = 0;
    if (!finalize(c, sd, sums(c.m, true), cfg, clamped)) return false;
    warn = std::max(violation, clamped) > cfg.scaling_tol;
    return true;
}

// ---- reduced Laplacians (block_elim/schur.rs) ----
struct Lap {  // symmetric CSR with explicit diagonal
    uint32_t n = 0;
    std::vector<uint32_t> ptr{0}, col;
    std::vector<double> val;
};

Lap exact_reduced(const Comp& c, const std::vector<double>& inv_e) {
    const uint32_t ne = c.m.nr(), nk = c.m.nc();
    std::vector<double> surplus(nk, 0.0);
    if (c.grounded) {
        for (uint32_t i = 0; i < nk; ++i) {
            double acc = c.ground[ne + i];
            for (uint32_t a = c.m.ct.ptr[i]; a < c.m.ct.ptr[i + 1]; ++a)
                acc += c.m.ct.val[a] * (inv_e[c.m.ct.col[a]] * c.ground[c.m.ct.col[a]]);
            surplus[i] = acc;
        }
    }
    Lap L;
    L.n = nk + (c.grounded ? 1 : 0);
    // row i of the reduced matrix depends only on the rows of C through the
    // neighbours of kept vertex i, so blocks of rows are formed on host
    // threads (each row by the same sequential loop) and joined in row order
    struct RowOut {
        std::vector<uint32_t> col;
        std::vector<double> val;
    };
    // the work of row i is the sum of the C-row lengths of its neighbours;
    // over all rows that is the sum of the squared C-row lengths
    uint64_t work_est = 0;
    for (uint32_t k = 0; k < ne; ++k) {
        const uint64_t len = c.m.c.ptr[k + 1] - c.m.c.ptr[k];
        work_est += len * len;
    }
    const uint32_t RBLK = nk >= 1024 ? 4 : 1;
    const uint32_t nblk = (nk + RBLK - 1) / RBLK;
    std::vector<std::vector<RowOut>> rows(nblk);
    auto row_block = [&](size_t bi) {
        std::vector<double> work(nk, 0.0);
        std::vector<uint32_t> touched;
        const uint32_t i0 = (uint32_t)bi * RBLK, i1 = std::min(nk, i0 + RBLK);
        rows[bi].resize(i1 - i0);
        for (uint32_t i = i0; i < i1; ++i) {
            RowOut& R = rows[bi][i - i0];
            work[i] = c.diag[ne + i];
            touched.push_back(i);
            for (uint32_t a = c.m.ct.ptr[i]; a < c.m.ct.ptr[i + 1]; ++a) {
                uint32_t k = c.m.ct.col[a];
                double w = c.m.ct.val[a], inv = inv_e[k];
                for (uint32_t b = c.m.c.ptr[k]; b < c.m.c.ptr[k + 1]; ++b) {
                    uint32_t j = c.m.c.col[b];
                    if (work[j] == 0.0 && j != i) touched.push_back(j);
                    work[j] -= (w * c.m.c.val[b]) * inv;
                }
            }
            std::sort(touched.begin(), touched.end());
            touched.erase(std::unique(touched.begin(), touched.end()), touched.end());
            double adjacency = 0;
            size_t dpos = 0;
            for (uint32_t j : touched) {
                double v = work[j];
                work[j] = 0.0;
                if (j == i) {
                    dpos = R.col.size();
                    R.col.push_back(j);
                    R.val.push_back(0.0);
                } else if (v != 0.0) {
                    adjacency -= v;
                    R.col.push_back(j);
                    R.val.push_back(v);
                }
            }
            R.val[dpos] = adjacency + surplus[i];
            if (c.grounded && surplus[i] > 0.0) {
                R.col.push_back(nk);
                R.val.push_back(-surplus[i]);
            }
            touched.clear();
        }
    };
    // worth threads only when the rows reach many eliminated neighbours
    if (c.m.c.nnz() >= (1u << 20) || work_est >= ((uint64_t)1 << 22)) par_for_each(nblk, row_block);
    else for (size_t bi = 0; bi < nblk; ++bi) row_block(bi);
    for (auto& blk : rows)
        for (RowOut& R : blk) {
            L.col.insert(L.col.end(), R.col.begin(), R.col.end());
            L.val.insert(L.val.end(), R.val.begin(), R.val.end());
            L.ptr.push_back((uint32_t)L.col.size());
        }
    if (c.grounded) {
        for (uint32_t i = 0; i < nk; ++i)
            if (surplus[i] > 0.0) {
                L.col.push_back(i);
                L.val.push_back(-surplus[i]);
            }
        L.col.push_back(nk);
        L.val.push_back(neumaier(surplus.data(), surplus.size()));
        L.ptr.push_back((uint32_t)L.col.size());
    }
    return L;
}

uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
struct Rng {
    uint64_t s;
    double unit() { s = mix64(s); return (double)(s >> 11) * (1.0 / 9007199254740992.0); }
};

struct Edge { uint32_t lo, hi; double w; };

// Clique-tree sample of one star (GKS): neighbours ascending by weight, each
// linked to a later one drawn in proportion to weight, weight w_i S_i / d.
// `split` > 1 first splits every neighbour edge into that many equal copies.
// `pre` is the caller's scratch for the weight prefix sums.
void sample_star(std::vector<std::pair<uint32_t, double>>& e, uint32_t split, Rng& rng,
                 std::vector<Edge>& out, std::vector<double>& pre) {
    if (split > 1) {
        std::vector<std::pair<uint32_t, double>> s;
        s.reserve(e.size() * split);
        for (auto& x : e)
            for (uint32_t k = 0; k < split; ++k) s.push_back({x.first, x.second / split});
        e.swap(s);
    }
    if (e.size() <= 1) return;
    std::sort(e.begin(), e.end(), [](const std::pair<uint32_t, double>& a, const std::pair<uint32_t, double>& b) {
        return a.second != b.second ? a.second < b.second : a.first < b.first;
    });
    const size_t m = e.size();
    pre.resize(m + 1);
    pre[0] = 0.0;
    for (size_t i = 0; i < m; ++i) pre[i + 1] = pre[i] + e[i].second;
    const double d = pre[m];
    for (size_t i = 0; i + 1 < m; ++i) {
        double S = d - pre[i + 1];
        if (!(S > 0.0)) continue;
        double tgt = pre[i + 1] + rng.unit() * S;
        size_t j = (size_t)(std::upper_bound(pre.begin() + i + 2, pre.begin() + m + 1, tgt) - pre.begin()) - 1;
        j = std::min(std::max(j, i + 1), m - 1);
        if (e[i].first == e[j].first) continue;
        out.push_back({std::min(e[i].first, e[j].first), std::max(e[i].first, e[j].first),
                       e[i].second * S / d});
    }
}

// Laplacian of a weighted edge list given as consecutive parts (the parts in
// order are the list).  Parallel edges are summed in ascending weight: the
// edges are bucketed by lo (per-chunk counts, so chunks of parts scatter on
// host threads; within a bucket the edges keep list order), each bucket is
// sorted by (hi, w) and its runs of equal hi summed in that order -- the order
// of one global sort on (lo, hi, w).
Lap lap_from_edges(std::vector<std::vector<Edge>>& parts, uint32_t n) {
    static const char* const steps[] = {"bucket", "sort and merge", "rows"};
    StepTimes st("edges to rows", steps, 3);
    size_t cap = std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
    if (const char* e = std::getenv("WITHIN_HOST_THREADS")) cap = std::max(1, std::atoi(e));
    size_t total = 0;
    for (auto& p : parts) total += p.size();
    // chunks: contiguous runs of parts with about total / nch edges each
    const size_t nch = total >= ((size_t)1 << 16) ? std::max<size_t>(1, std::min(cap, parts.size())) : 1;
    std::vector<size_t> ch_part{0};
    {
        size_t acc = 0, goal = (total + nch - 1) / nch;
        for (size_t p = 0; p < parts.size(); ++p) {
            acc += parts[p].size();
            if (acc >= goal * ch_part.size() && ch_part.size() < nch) ch_part.push_back(p + 1);
        }
        while (ch_part.size() <= nch) ch_part.push_back(parts.size());
    }
    std::vector<std::vector<uint32_t>> cnt(nch);
    par_for_each(nch, [&](size_t t) {
        cnt[t].assign(n, 0);
        for (size_t p = ch_part[t]; p < ch_part[t + 1]; ++p)
            for (const Edge& e : parts[p]) ++cnt[t][e.lo];
    });
    std::vector<uint32_t> start(n + 1, 0);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t s0 = start[i];
        for (size_t t = 0; t < nch; ++t) {
            const uint32_t c = cnt[t][i];
            cnt[t][i] = s0;   // now: where chunk t's first edge of bucket i goes
            s0 += c;
        }
        start[i + 1] = s0;
    }
    std::vector<Edge> srt(total);
    par_for_each(nch, [&](size_t t) {
        std::vector<uint32_t>& pos = cnt[t];
        for (size_t p = ch_part[t]; p < ch_part[t + 1]; ++p) {
            for (const Edge& e : parts[p]) srt[pos[e.lo]++] = e;
            std::vector<Edge>().swap(parts[p]);
        }
        std::vector<uint32_t>().swap(pos);
    });
    st.mark(0);
    // each bucket sorts and merges on its own (blocks of buckets on host threads)
    std::vector<uint32_t> kept(n, 0);
    const uint32_t gblk = 256;
    par_for_each(((size_t)n + gblk - 1) / gblk, [&](size_t b) {
        const uint32_t i1 = (uint32_t)std::min<size_t>(n, (b + 1) * (size_t)gblk);
        for (uint32_t i = (uint32_t)(b * gblk); i < i1; ++i) {
            Edge* g0 = srt.data() + start[i];
            Edge* g1 = srt.data() + start[i + 1];
            std::sort(g0, g1, [](const Edge& a, const Edge& b2) {
                if (a.hi != b2.hi) return a.hi < b2.hi;
                return a.w < b2.w;
            });
            Edge* w = g0;
            for (Edge* e = g0; e < g1; ++e) {
                if (w != g0 && (w - 1)->hi == e->hi) (w - 1)->w += e->w;
                else *w++ = *e;
            }
            kept[i] = (uint32_t)(w - g0);
        }
    });
    st.mark(1);
    // rows in one flat array sorted by column without a sort: the merged
    // edges are ordered by (lo, hi), so the edges reaching row i from below
    // (hi == i) arrive in ascending lo and those leaving it upwards (lo == i,
    // bucket i) in ascending hi; row i is [lower neighbours, i, upper
    // neighbours], its diagonal the sum of the lower then the upper weights
    // (the order one pass over the merged list adds them).  Lower entries are
    // scattered by chunks of buckets (contiguous lo ranges, per-chunk counts),
    // so every row receives them in ascending lo.
    std::vector<uint32_t> bch{0};   // chunk t = buckets [bch[t], bch[t+1])
    {
        uint64_t merged = 0;
        for (uint32_t g = 0; g < n; ++g) merged += kept[g];
        const size_t nrc = merged >= ((uint64_t)1 << 16) ? std::max<size_t>(1, cap) : 1;
        const uint64_t goal = (merged + nrc - 1) / nrc;
        uint64_t acc = 0;
        for (uint32_t g = 0; g < n; ++g) {
            acc += kept[g];
            if (acc >= goal * bch.size() && bch.size() < nrc) bch.push_back(g + 1);
        }
        while (bch.back() != n) bch.push_back(n);
    }
    const size_t nrc = bch.size() - 1;
    std::vector<std::vector<uint32_t>> lowc(nrc);
    par_for_each(nrc, [&](size_t t) {
        lowc[t].assign(n, 0);
        for (uint32_t g = bch[t]; g < bch[t + 1]; ++g)
            for (uint32_t q = start[g]; q < start[g] + kept[g]; ++q) ++lowc[t][srt[q].hi];
    });
    std::vector<uint32_t> rp(n + 1, 0), nlow(n, 0);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t l = 0;
        for (size_t t = 0; t < nrc; ++t) {
            const uint32_t c = lowc[t][i];
            lowc[t][i] = rp[i] + l;   // now: where chunk t's first lower entry of row i goes
            l += c;
        }
        nlow[i] = l;
        rp[i + 1] = rp[i] + l + 1 + kept[i];
    }
    Lap L;
    L.n = n;
    L.col.resize(rp[n]);
    L.val.resize(rp[n]);
    L.ptr.assign(rp.begin(), rp.end());
    par_for_each(nrc, [&](size_t t) {
        std::vector<uint32_t>& pos = lowc[t];
        for (uint32_t g = bch[t]; g < bch[t + 1]; ++g) {
            uint32_t up = rp[g] + nlow[g] + 1;
            for (uint32_t q = start[g]; q < start[g] + kept[g]; ++q) {
                const Edge& e = srt[q];
                const uint32_t b = pos[e.hi]++;
                L.col[b] = e.lo;
                L.val[b] = -e.w;
                L.col[up] = e.hi;
                L.val[up] = -e.w;
                ++up;
            }
        }
        std::vector<uint32_t>().swap(pos);
    });
    const uint32_t rblk = 4096;
    par_for_each(((size_t)n + rblk - 1) / rblk, [&](size_t b) {
        const uint32_t i1 = (uint32_t)std::min<size_t>(n, (b + 1) * (size_t)rblk);
        for (uint32_t i = (uint32_t)(b * rblk); i < i1; ++i) {
            const uint32_t q = rp[i] + nlow[i];
            double d = 0.0;
            for (uint32_t a = rp[i]; a < q; ++a) d += -L.val[a];
            for (uint32_t a = q + 1; a < rp[i + 1]; ++a) d += -L.val[a];
            L.col[q] = i;
            L.val[q] = d;
        }
    });
    st.mark(2);
    return L;
}

Lap sampled_reduced(const Comp& c, uint64_t seed, uint32_t split) {
    const uint32_t ne = c.m.nr(), nk = c.m.nc();
    // every eliminated vertex draws from its own seeded stream, so blocks of
    // vertices sample on host threads; the blocks' edge lists, in vertex
    // order, are the list of one sequential pass
    const uint32_t block = 2048;
    const size_t nblk = ((size_t)ne + block - 1) / block;
    std::vector<std::vector<Edge>> part(nblk + 1);
    par_for_each(nblk, [&](size_t b) {
        std::vector<std::pair<uint32_t, double>> ent;
        std::vector<double> pre;
        std::vector<Edge>& out = part[b];
        const uint32_t k1 = (uint32_t)std::min<size_t>(ne, (b + 1) * (size_t)block);
        out.reserve((size_t)(c.m.c.ptr[k1] - c.m.c.ptr[(uint32_t)(b * block)]));
        for (uint32_t k = (uint32_t)(b * block); k < k1; ++k) {
            ent.clear();
            for (uint32_t a = c.m.c.ptr[k]; a < c.m.c.ptr[k + 1]; ++a) ent.push_back({c.m.c.col[a], c.m.c.val[a]});
            if (ent.empty()) continue;
            if (c.grounded && c.ground[k] > 0.0) ent.push_back({nk, c.ground[k]});
            if (ent.size() <= 1) continue;
            Rng r{mix64(seed * 0x100000001B3ull + k)};
            sample_star(ent, split, r, out, pre);
        }
    });
    if (c.grounded)
        for (uint32_t i = 0; i < nk; ++i)
            if (c.ground[ne + i] > 0.0) part[nblk].push_back({i, nk, c.ground[ne + i]});
    return lap_from_edges(part, nk + (c.grounded ? 1 : 0));
}

// ---- factors of a reduced Laplacian ----
struct Factor {
    uint32_t n = 0;
    bool dense = false;
    std::vector<double> pinv;                 // dense generalised inverse, n x n
    std::vector<uint32_t> round;              // per vertex: elimination round
    std::vector<double> dinv;                 // per vertex
    std::vector<std::vector<std::pair<uint32_t, double>>> colv;  // per vertex: (later row, l)
    uint32_t n_rounds = 0;
    // the vertices left when the rounds stop (see ac_rounds): with core_dense
    // their Schur complement is applied as a dense generalised inverse
    // core_pinv (core.size()^2, row-major over `core`), otherwise by its diagonal.
    std::vector<uint32_t> core;
    bool core_dense = false;
    std::vector<double> core_pinv;
};

// Dense LDL^T in natural order with pseudo-inverse pivots, materialised as
// G = L^-T D^+ L^-1.  Returns false on a clearly negative pivot.  Laid out
// for the cache and the vector units: the factorisation updates the lower
// triangle row by row (contiguous), L^-1 is formed row by row from earlier
// rows, and the rows of G are independent sums spread over host threads.
bool dense_pinv(const Lap& m, Factor& f) {
    const uint32_t n = m.n;
    std::vector<double> a((size_t)n * n, 0.0);   // lower triangle (row-major) used
    double maxd = 0;
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t k = m.ptr[i]; k < m.ptr[i + 1]; ++k) {
            a[(size_t)i * n + m.col[k]] += m.val[k];
            if (m.col[k] == i) maxd = std::max(maxd, std::fabs(m.val[k]));
        }
    const double fl = 1e-13 * std::max(maxd, DBL_MIN) * std::max<uint32_t>(n, 1);
    std::vector<double> piv(n, 0.0), c(n);
    for (uint32_t k = 0; k < n; ++k) {
        const double d = a[(size_t)k * n + k];
        if (d < -fl) return false;
        if (d <= fl) {
            piv[k] = 0.0;
            for (uint32_t i = k + 1; i < n; ++i) a[(size_t)i * n + k] = 0.0;
            continue;
        }
        piv[k] = d;
        const double inv = 1.0 / d;
        for (uint32_t i = k + 1; i < n; ++i) c[i] = a[(size_t)i * n + k];   // column k, before scaling
        for (uint32_t i = k + 1; i < n; ++i) {
            const double ci = c[i];
            if (ci == 0.0) continue;
            const double li = ci * inv;
            double* row = &a[(size_t)i * n];
            for (uint32_t j = k + 1; j <= i; ++j) row[j] -= li * c[j];
            row[k] = li;   // L below the diagonal
        }
    }
    // L^-1 (unit lower), row i from the rows before it: Li[i] = e_i - sum_k L[i][k] Li[k]
    std::vector<double> li((size_t)n * n, 0.0);
    for (uint32_t i = 0; i < n; ++i) {
        double* ri = &li[(size_t)i * n];
        ri[i] = 1.0;
        const double* lrow = &a[(size_t)i * n];
        for (uint32_t k = 0; k < i; ++k) {
            const double l = lrow[k];
            if (l == 0.0) continue;
            const double* rk = &li[(size_t)k * n];
            for (uint32_t j = 0; j <= k; ++j) ri[j] -= l * rk[j];
        }
    }
    // G[r][c] = sum_k D^+_k Li[k][r] Li[k][c] (k >= max(r, c)), one row of G per task
    f.n = n;
    f.dense = true;
    f.pinv.assign((size_t)n * n, 0.0);
    std::vector<double> dp(n);
    for (uint32_t k = 0; k < n; ++k) dp[k] = piv[k] > 0.0 ? 1.0 / piv[k] : 0.0;
    par_for_each(n, [&](size_t r) {
        double* g = &f.pinv[r * n];
        for (uint32_t k = (uint32_t)r; k < n; ++k) {
            const double* rk = &li[(size_t)k * n];
            const double w = dp[k] * rk[r];
            if (w == 0.0) continue;
            for (uint32_t cc = 0; cc <= k; ++cc) g[cc] += w * rk[cc];
        }
    });
    // symmetrise the roundoff
    for (uint32_t r = 0; r < n; ++r)
        for (uint32_t cc = r + 1; cc < n; ++cc) {
            double v = 0.5 * (f.pinv[(size_t)r * n + cc] + f.pinv[(size_t)cc * n + r]);
            f.pinv[(size_t)r * n + cc] = v;
            f.pinv[(size_t)cc * n + r] = v;
        }
    return true;
}

// Round-parallel approximate Cholesky of a Laplacian.  Each round eliminates an
// independent set: vertices whose (capped degree, hash, id) key is smaller than
// every alive neighbour's.  Low-degree vertices therefore go first, which keeps
// fill low; the clique of an eliminated vertex is replaced by a sampled tree.
void ac_rounds(const Lap& m, const PrecondCfg& cfg, Factor& f) {
    const uint64_t seed = cfg.ac_seed;
    const uint32_t split = cfg.ac_split;
    const uint32_t n = m.n;
    static const char* const steps[] = {"adjacency", "compact", "core", "select", "eliminate", "fill"};
    StepTimes st("rounds", steps, 6);
    std::vector<std::vector<std::pair<uint32_t, double>>> adj(n);
    par_for_each(((size_t)n + 4095) / 4096, [&](size_t b) {
        const uint32_t i1 = (uint32_t)std::min<size_t>(n, (b + 1) * (size_t)4096);
        for (uint32_t i = (uint32_t)(b * 4096); i < i1; ++i) {
            uint32_t c = 0;
            for (uint32_t k = m.ptr[i]; k < m.ptr[i + 1]; ++k) c += m.col[k] != i && m.val[k] < 0.0;
            adj[i].reserve(c);
            for (uint32_t k = m.ptr[i]; k < m.ptr[i + 1]; ++k)
                if (m.col[k] != i && m.val[k] < 0.0) adj[i].push_back({m.col[k], -m.val[k]});
        }
    });
    f.n = n;
    f.dense = false;
    f.round.assign(n, 0);
    f.dinv.assign(n, 0.0);
    f.colv.assign(n, {});
    std::vector<char> alive(n, 1);
    std::vector<uint32_t> sorted_len(n, 0);   // see the compaction below
    std::vector<uint32_t> live(n);
    std::iota(live.begin(), live.end(), 0u);
    std::vector<uint64_t> key(n);
    std::vector<uint32_t> sel;
    uint32_t r = 0;
    double last_frac = 1.0;
    bool dense_graph = false;   // see the stop rules below
    // Every vertex's compaction, key, selection test and elimination reads
    // only its own adjacency (and its neighbours' keys), and every eliminated
    // vertex samples from its own seeded stream, so these run over blocks of
    // vertices on host threads; selections and fill edges are joined in
    // vertex order, which gives the sequential loop's lists exactly.
    // A large graph runs in blocks of 4096 vertices, a smaller one (a
    // reduced system of a few thousand levels, whose rounds fill it in) in
    // blocks of about n / 64.  The block size only schedules work.
    const bool threaded = n >= 1024;
    const size_t VBLK = n >= 16384 ? 4096 : std::max<size_t>(32, ((size_t)n + 63) / 64);
    auto blocks = [VBLK](size_t k) { return (k + VBLK - 1) / VBLK; };
    auto par = [&](size_t nb, auto&& fn) {
        if (threaded) par_for_each(nb, fn);
        else for (size_t b = 0; b < nb; ++b) fn(b);
    };
    st.mark(0);
    while (!live.empty()) {
        // compact adjacency: drop dead neighbours, merge parallel edges.  A
        // list is [sorted prefix: one entry per neighbour, ascending, from the
        // last compaction | fill edges appended since]; the tail is sorted
        // stably by neighbour and merged in, each neighbour's weight summed as
        // prefix entry first, then its tail entries in append order (the
        // order of one accumulation pass over the list).
        par(blocks(live.size()), [&](size_t b) {
            std::vector<std::pair<uint32_t, double>> tail, merged;
            const size_t j1 = std::min(live.size(), (b + 1) * VBLK);
            for (size_t j = b * VBLK; j < j1; ++j) {
                const uint32_t v = live[j];
                auto& a = adj[v];
                const size_t s0 = sorted_len[v];
                if (s0 == a.size()) {
                    size_t w = 0;
                    for (auto& e : a)
                        if (alive[e.first] && e.first != v) a[w++] = e;
                    a.resize(w);
                } else {
                    tail.clear();
                    for (size_t q = s0; q < a.size(); ++q)
                        if (alive[a[q].first] && a[q].first != v) tail.push_back(a[q]);
                    std::stable_sort(tail.begin(), tail.end(),
                                     [](const std::pair<uint32_t, double>& x, const std::pair<uint32_t, double>& y) {
                                         return x.first < y.first;
                                     });
                    merged.clear();
                    size_t p = 0, t = 0;
                    while (p < s0 || t < tail.size()) {
                        if (p < s0 && (!alive[a[p].first] || a[p].first == v)) {
                            ++p;
                            continue;
                        }
                        uint32_t u;
                        double acc;
                        if (p < s0 && (t >= tail.size() || a[p].first <= tail[t].first)) {
                            u = a[p].first;
                            acc = a[p].second;
                            ++p;
                        } else {
                            u = tail[t].first;
                            acc = tail[t].second;
                            ++t;
                        }
                        for (; t < tail.size() && tail[t].first == u; ++t) acc += tail[t].second;
                        merged.push_back({u, acc});
                    }
                    a.assign(merged.begin(), merged.end());
                }
                sorted_len[v] = (uint32_t)a.size();
                uint64_t deg = std::min<uint64_t>(a.size(), 255);
                key[v] = (deg << 56) | (mix64(seed ^ ((uint64_t)v << 20) ^ r) & 0x00FFFFFFFF000000ull) | 0;
            }
        });
        st.mark(1);
        // Stop the rounds once the remaining graph is a small or dense core:
        // a dense core (<= core_dense_max vertices) is inverted exactly; a
        // larger one, reached when rounds stop paying (fewer than
        // core_min_frac of the vertices eliminated) or at max_rounds, keeps
        // only its diagonal -- its intra-core edges are dropped, which leaves
        // an SDD (positive semi-definite) approximation of the core.
        // A graph whose rounds stall while nearly all of it is still alive
        // (more than DENSE_ALIVE of the vertices: a few thousand kept levels
        // with a dense or banded Schur complement, where every round removes
        // only a few per cent) and that has at most core_small vertices keeps
        // eliminating until core_dense_late remain: its diagonal alone would
        // leave almost the whole reduced system approximated by its diagonal.
        // A graph that stalls after its rounds removed a good part of it (the
        // worker/firm panels) stops as before.
        constexpr double DENSE_ALIVE = 0.8;
        const bool plain_stall = last_frac < cfg.core_min_frac || r >= cfg.max_rounds;
        if (!dense_graph && plain_stall && r > 0 && live.size() <= cfg.core_small &&
            (double)live.size() > DENSE_ALIVE * (double)n)
            dense_graph = true;
        const uint32_t dense_at =
            dense_graph ? std::min(cfg.core_dense_max, cfg.core_dense_late) : cfg.core_dense_max;
        const bool small = live.size() <= dense_at && live.size() > 1;
        const bool stalled = dense_graph ? (last_frac < cfg.core_min_frac_small || r >= 4 * cfg.max_rounds)
                                         : plain_stall;
        if (small || (stalled && live.size() > 1)) {
            f.core = live;
            std::sort(f.core.begin(), f.core.end());
            for (uint32_t v : f.core) f.round[v] = r;
            if (small) {
                f.core_dense = true;
                std::vector<uint32_t> pos(n, UINT32_MAX);
                for (uint32_t i = 0; i < f.core.size(); ++i) pos[f.core[i]] = i;
                Lap c;
                c.n = (uint32_t)f.core.size();
                for (uint32_t i = 0; i < c.n; ++i) {
                    double deg = 0;
                    std::vector<std::pair<uint32_t, double>> row;
                    for (auto& e : adj[f.core[i]]) {
                        row.push_back({pos[e.first], -e.second});
                        deg += e.second;
                    }
                    row.push_back({i, deg});
                    std::sort(row.begin(), row.end());
                    for (auto& x : row) {
                        c.col.push_back(x.first);
                        c.val.push_back(x.second);
                    }
                    c.ptr.push_back((uint32_t)c.col.size());
                }
                Factor cf;
                if (!dense_pinv(c, cf)) throw WError(ERR_SINGULAR, "dense core factorisation failed");
                f.core_pinv = std::move(cf.pinv);
                for (uint32_t v : f.core) f.dinv[v] = 0.0;   // forward pass only; the core mat-vec writes x
            } else {
                f.core_dense = false;
                for (uint32_t v : f.core) {
                    double d = 0;
                    for (auto& e : adj[v]) d += e.second;
                    f.dinv[v] = d > 0.0 ? 1.0 / d : 0.0;
                }
            }
            ++r;
            st.mark(2);
            break;
        }
        st.mark(2);
        // the round: every live vertex that is the minimum of (key, id) over its neighbours
        std::vector<std::vector<uint32_t>> sel_part(blocks(live.size()));
        par(sel_part.size(), [&](size_t b) {
            const size_t j1 = std::min(live.size(), (b + 1) * VBLK);
            for (size_t j = b * VBLK; j < j1; ++j) {
                const uint32_t v = live[j];
                bool best = true;
                for (auto& e : adj[v]) {
                    uint32_t u = e.first;
                    if (key[u] < key[v] || (key[u] == key[v] && u < v)) {
                        best = false;
                        break;
                    }
                }
                if (best) sel_part[b].push_back(v);
            }
        });
        sel.clear();
        for (auto& p : sel_part) sel.insert(sel.end(), p.begin(), p.end());
        st.mark(3);
        // eliminate the round: columns of L, pivots and sampled fill edges
        // (a dense graph's rounds select few vertices of high degree: small blocks)
        const size_t EBLK = n >= 16384 ? VBLK : 4;
        std::vector<std::vector<Edge>> fill_part((sel.size() + EBLK - 1) / EBLK);
        par(fill_part.size(), [&](size_t b) {
            std::vector<std::pair<uint32_t, double>> ent;
            std::vector<double> pre;
            const size_t j1 = std::min(sel.size(), (b + 1) * EBLK);
            for (size_t j = b * EBLK; j < j1; ++j) {
                const uint32_t v = sel[j];
                f.round[v] = r;
                double d = 0;
                for (auto& e : adj[v]) d += e.second;
                if (!(d > 0.0)) {
                    f.dinv[v] = 0.0;
                    continue;
                }
                f.dinv[v] = 1.0 / d;
                auto& cv = f.colv[v];
                for (auto& e : adj[v]) cv.push_back({e.first, -e.second / d});
                ent = adj[v];
                Rng rng{mix64(seed * 0x9E3779B97F4A7C15ull + v + 1)};
                sample_star(ent, split, rng, fill_part[b], pre);
            }
        });
        st.mark(4);
        for (uint32_t v : sel) {
            alive[v] = 0;
            adj[v].clear();
            adj[v].shrink_to_fit();
        }
        // append every fill edge to both endpoints' lists in fill order (the
        // parts in order are the fill list): chunks of parts count their
        // entries per vertex, then scatter them into a flat array by
        // (vertex, chunk), and blocks of vertices append their runs
        {
            size_t n_fill = 0;
            for (auto& p : fill_part) n_fill += p.size();
            size_t nch = 1;
            if (threaded && n_fill >= 4096)
                nch = std::min<size_t>({(size_t)16, fill_part.size(), std::max<size_t>(1, 2 * n_fill / n)});
            if (nch <= 1) {
                for (auto& p : fill_part)
                    for (auto& e : p) {
                        adj[e.lo].push_back({e.hi, e.w});
                        adj[e.hi].push_back({e.lo, e.w});
                    }
            } else {
                std::vector<size_t> cp{0};
                {
                    size_t acc = 0, goal = (n_fill + nch - 1) / nch;
                    for (size_t q = 0; q < fill_part.size(); ++q) {
                        acc += fill_part[q].size();
                        if (acc >= goal * cp.size() && cp.size() < nch) cp.push_back(q + 1);
                    }
                    while (cp.size() <= nch) cp.push_back(fill_part.size());
                }
                std::vector<std::vector<uint32_t>> cnt(nch);
                par_for_each(nch, [&](size_t t) {
                    cnt[t].assign(n, 0);
                    for (size_t q = cp[t]; q < cp[t + 1]; ++q)
                        for (auto& e : fill_part[q]) {
                            ++cnt[t][e.lo];
                            ++cnt[t][e.hi];
                        }
                });
                std::vector<size_t> beg(n + 1, 0);
                for (uint32_t u = 0; u < n; ++u) {
                    size_t o = beg[u];
                    for (size_t t = 0; t < nch; ++t) {
                        const uint32_t c = cnt[t][u];
                        cnt[t][u] = (uint32_t)(o - beg[u]);   // chunk t's first entry within u's run
                        o += c;
                    }
                    beg[u + 1] = o;
                }
                std::vector<std::pair<uint32_t, double>> flat(beg[n]);
                par_for_each(nch, [&](size_t t) {
                    std::vector<uint32_t>& pos = cnt[t];
                    for (size_t q = cp[t]; q < cp[t + 1]; ++q)
                        for (auto& e : fill_part[q]) {
                            flat[beg[e.lo] + pos[e.lo]++] = {e.hi, e.w};
                            flat[beg[e.hi] + pos[e.hi]++] = {e.lo, e.w};
                        }
                });
                par_for_each(((size_t)n + 4095) / 4096, [&](size_t b) {
                    const uint32_t u1 = (uint32_t)std::min<size_t>(n, (b + 1) * (size_t)4096);
                    for (uint32_t u = (uint32_t)(b * 4096); u < u1; ++u)
                        if (beg[u + 1] > beg[u])
                            adj[u].insert(adj[u].end(), flat.begin() + beg[u], flat.begin() + beg[u + 1]);
                });
            }
        }
        const size_t before = live.size();
        size_t w = 0;
        for (uint32_t v : live)
            if (alive[v]) live[w++] = v;
        live.resize(w);
        last_frac = (double)sel.size() / (double)before;
        ++r;
        st.mark(5);
    }
    f.n_rounds = r;
}

void factor_lap(const Lap& L, const PrecondCfg& cfg, Factor& f) {
    if (L.n <= DENSE_MAX && dense_pinv(L, f)) return;
    ac_rounds(L, cfg, f);
}

// Gremban cover of a signed matrix (block_elim/solver.rs:220-271).
Comp cover_of(const Comp& c) {
    const Csr& a = c.m.c;
    const uint32_t nr = a.nr, nc = a.nc;
    Comp o;
    o.m.c.nr = 2 * nr;
    o.m.c.nc = 2 * nc;
    for (int copy = 0; copy < 2; ++copy)
        for (uint32_t i = 0; i < nr; ++i) {
            for (int cs = 0; cs < 2; ++cs) {
                uint32_t base = cs ? nc : 0;
                bool neg = (cs != 0) != (copy != 0);
                for (uint32_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
                    double v = a.val[k];
                    if ((v < 0.0) != neg) continue;
                    o.m.c.col.push_back(a.col[k] + base);
                    o.m.c.val.push_back(std::fabs(v));
                }
            }
            o.m.c.ptr.push_back((uint32_t)o.m.c.col.size());
        }
    o.m.ct = transpose(o.m.c);
    auto dbl = [&](const std::vector<double>& v) {
        std::vector<double> r;
        r.insert(r.end(), v.begin(), v.begin() + nr);
        r.insert(r.end(), v.begin(), v.begin() + nr);
        r.insert(r.end(), v.begin() + nr, v.end());
        r.insert(r.end(), v.begin() + nr, v.end());
        return r;
    };
    o.diag = dbl(c.diag);
    o.ground = dbl(c.ground);
    o.grounded = c.grounded;
    o.laplacian = true;
    return o;
}

std::vector<double> inv_elim(const Comp& c) {
    std::vector<double> inv(c.m.nr());
    for (uint32_t i = 0; i < c.m.nr(); ++i) {
        if (!(c.diag[i] > 0.0)) throw WError(ERR_SINGULAR, "zero diagonal in preconditioner at index " + std::to_string(i));
        inv[i] = 1.0 / c.diag[i];
    }
    return inv;
}

// LocalSolverConfig routing of factor_reduced (block_elim/solver.rs:191-217):
// exact reduced system when n_kept <= dense_threshold or SchurMode::Exact,
// otherwise the clique-tree sampled one.
Lap reduced_for(const Comp& c, const std::vector<double>& inv_e, const PrecondCfg& cfg) {
    bool exact = cfg.schur_exact || (cfg.dense_threshold > 0 && c.m.nc() <= cfg.dense_threshold);
    return exact ? exact_reduced(c, inv_e) : sampled_reduced(c, cfg.schur_seed, std::max(1u, cfg.schur_split));
}

struct Domain {
    std::vector<uint32_t> globals;
    std::vector<double> pw;
    Comp comp;
    std::vector<double> inv_e;
    Factor fac;
    int mode = 0;   // 0 floating, 1 grounded, 2 cover
};

}  // namespace

// ---------------------------------------------------------------------------
std::vector<ChannelPair> schwarz_channel_pairs(const HostDesign& d) {
    std::vector<std::pair<uint32_t, int>> ch;   // (term, load index or -1)
    for (uint32_t t = 0; t < d.terms.size(); ++t)
        for (int c : d.terms[t].cols) ch.push_back({t, c});
    std::vector<ChannelPair> out;
    for (size_t a = 0; a < ch.size(); ++a)
        for (size_t b = a + 1; b < ch.size(); ++b)
            if (ch[a].first != ch[b].first) out.push_back({ch[a].first, ch[b].first, ch[a].second, ch[b].second});
    return out;
}

BuildResult build_preconditioner(const HostDesign& d, const double* w, const PrecondCfg& cfg,
                                 std::vector<CrossTab>* cross_tabs,
                                 const std::vector<std::shared_future<void>>* ready) {
    BuildResult out;
    if (cfg.kind == 0) return out;
    if (cfg.kind == 2) {  // operator/schwarz.rs:185-229
        out.kind = 2;
        out.inv_diag.assign(d.n_dofs, 0.0);
        for (size_t q = 0; q < d.terms.size(); ++q) {
            const Term& t = d.terms[q];
            const uint32_t* lv = d.codes[q].data();
            for (size_t c = 0; c < t.cols.size(); ++c) {
                double* sl = &out.inv_diag[t.offset + c * t.n_levels];
                int k = t.cols[c];
                for (uint64_t i = 0; i < d.n_obs; ++i) {
                    double wi = w ? w[i] : 1.0;
                    sl[lv[i]] += k < 0 ? wi : wi * d.loads[k][i] * d.loads[k][i];
                }
            }
        }
        for (size_t i = 0; i < out.inv_diag.size(); ++i) {
            double& v = out.inv_diag[i];
            if (v == 0.0) continue;
            double inv = 1.0 / v;
            if (!std::isfinite(inv)) throw WError(ERR_SINGULAR, "zero diagonal in preconditioner at index " + std::to_string(i));
            v = inv;
        }
        return out;
    }

    // ---- additive Schwarz: subdomains (domain/factor_pairs.rs:36-152) ----
    struct Ch { uint32_t term, col; };
    std::vector<Ch> ch;
    for (uint32_t t = 0; t < d.terms.size(); ++t)
        for (uint32_t c = 0; c < d.terms[t].cols.size(); ++c) ch.push_back({t, c});
    bool any_slope = false;
    for (auto& x : ch) any_slope = any_slope || d.terms[x.term].cols[x.col] >= 0;
    // the levels that occur, per term: chunks of observations mark their own
    // copy, merged by blocks of levels (all on the host pool)
    std::vector<std::vector<char>> active(d.terms.size());
    for (size_t t = 0; t < d.terms.size(); ++t) {
        const uint32_t L = d.terms[t].n_levels;
        const uint32_t* cd = d.codes[t].data();
        const uint64_t n = d.n_obs;
        const size_t nch = n >= ((uint64_t)1 << 20) && (uint64_t)L * 16 <= ((uint64_t)1 << 28) ? 16 : 1;
        if (nch == 1) {
            active[t].assign(L, 0);
            for (uint64_t i = 0; i < n; ++i) active[t][cd[i]] = 1;
            continue;
        }
        const uint64_t per = (n + nch - 1) / nch;
        std::vector<std::vector<char>> part(nch);
        par_for_each(nch, [&](size_t c) {
            part[c].assign(L, 0);
            const uint64_t i1 = std::min(n, (c + 1) * per);
            for (uint64_t i = c * per; i < i1; ++i) part[c][cd[i]] = 1;
        });
        active[t].assign(L, 0);
        const size_t B = 1 << 16;
        par_for_each(((size_t)L + B - 1) / B, [&](size_t b) {
            const size_t l1 = std::min<size_t>(L, (b + 1) * B);
            for (size_t l = b * B; l < l1; ++l) {
                char a = 0;
                for (size_t c = 0; c < nch; ++c) a |= part[c][l];
                active[t][l] = a;
            }
        });
    }
    // channel pairs of different terms, each built on its own host thread
    // and concatenated in pair order
    std::vector<std::pair<size_t, size_t>> pairs;
    for (size_t a = 0; a < ch.size(); ++a)
        for (size_t b = a + 1; b < ch.size(); ++b)
            if (ch[a].term != ch[b].term) pairs.push_back({a, b});
    std::vector<std::vector<Domain>> pair_doms(pairs.size());
    std::vector<uint64_t> pair_warnings(pairs.size(), 0);
    BuildTrace tr_pairs("channel pairs: cross-tabs, components, SDDM forms");
    par_for_each(pairs.size(), [&](size_t pi) {
            BuildTrace tr_pair("pair", (long)pi);
            static const char* const psteps[] = {"maps", "cells", "diagonals", "labels"};
            StepTimes pst("pair set-up", psteps, 4);
            std::vector<Domain>& doms = pair_doms[pi];
            uint64_t& n_warnings = pair_warnings[pi];
            Ch R = ch[pairs[pi].first], Cc = ch[pairs[pi].second];
            const Term& TR = d.terms[R.term];
            const Term& TC = d.terms[Cc.term];
            std::vector<uint32_t> rmap(TR.n_levels, UINT32_MAX), cmap(TC.n_levels, UINT32_MAX), l2g;
            uint32_t nr = 0, nc = 0;
            for (uint32_t j = 0; j < TR.n_levels; ++j)
                if (active[R.term][j]) { rmap[j] = nr++; l2g.push_back(TR.offset + R.col * TR.n_levels + j); }
            for (uint32_t k = 0; k < TC.n_levels; ++k)
                if (active[Cc.term][k]) { cmap[k] = nc++; l2g.push_back(TC.offset + Cc.col * TC.n_levels + k); }
            if (nr == 0 || nc == 0) return;
            pst.mark(0);
            // weighted cross-tab, each cell summed in observation order (accumulate.rs)
            const uint32_t* rl = d.codes[R.term].data();
            const uint32_t* cl = d.codes[Cc.term].data();
            int kr = TR.cols[R.col], kc = TC.cols[Cc.col];
            std::vector<double> rdiag(nr, 0.0), cdiag(nc, 0.0);
            Bip full;
            full.c.nr = nr;
            full.c.nc = nc;
            if (cross_tabs) {
                // the GPU cross-tab over raw level ids: keep the active levels
                // (every cell's levels are active) and renumber them
                if (ready) (*ready)[pi].get();
                CrossTab& X = (*cross_tabs)[pi];
                if (nr == TR.n_levels && nc == TC.n_levels) {
                    // every level is active: the renumbering is the identity
                    full.c.ptr = std::move(X.row_ptr);
                    full.c.col = std::move(X.col);
                    full.c.val = std::move(X.val);
                    full.ct.nr = nc;
                    full.ct.nc = nr;
                    full.ct.ptr = std::move(X.col_ptr);
                    full.ct.col = std::move(X.row);
                    full.ct.val = std::move(X.tval);
                } else {
                    // the active levels' rows (every cell of one is kept), renumbered;
                    // rows copied by blocks on the host pool
                    auto renumber = [&](const std::vector<char>& act, uint32_t n_levels,
                                        const std::vector<uint32_t>& xptr, const std::vector<uint32_t>& xidx,
                                        const std::vector<double>& xval, const std::vector<uint32_t>& map,
                                        Csr& o) {
                        std::vector<uint32_t> src;
                        for (uint32_t j = 0; j < n_levels; ++j)
                            if (act[j]) src.push_back(j);
                        o.ptr.assign(src.size() + 1, 0);
                        for (size_t i = 0; i < src.size(); ++i)
                            o.ptr[i + 1] = o.ptr[i] + (xptr[src[i] + 1] - xptr[src[i]]);
                        o.col.resize(o.ptr.back());
                        o.val.resize(o.ptr.back());
                        const size_t RB = 16384;
                        par_for_each((src.size() + RB - 1) / RB, [&](size_t b) {
                            const size_t i1 = std::min(src.size(), (b + 1) * RB);
                            for (size_t i = b * RB; i < i1; ++i) {
                                uint32_t q = o.ptr[i];
                                for (uint32_t p = xptr[src[i]]; p < xptr[src[i] + 1]; ++p, ++q) {
                                    o.col[q] = map[xidx[p]];
                                    o.val[q] = xval[p];
                                }
                            }
                        });
                    };
                    renumber(active[R.term], TR.n_levels, X.row_ptr, X.col, X.val, cmap, full.c);
                    full.ct.nr = nc;
                    full.ct.nc = nr;
                    renumber(active[Cc.term], TC.n_levels, X.col_ptr, X.row, X.tval, rmap, full.ct);
                }
                pst.mark(1);
                if (!w && kr < 0 && kc < 0) {
                    // unweighted intercepts: the diagonals are observation counts,
                    // integer sums of the cells (exact in any order)
                    auto row_sums = [&](const Csr& m, std::vector<double>& out) {
                        const uint32_t RB = 16384;
                        par_for_each(((size_t)m.nr + RB - 1) / RB, [&](size_t b) {
                            const uint32_t r1 = (uint32_t)std::min<size_t>(m.nr, (b + 1) * (size_t)RB);
                            for (uint32_t r = (uint32_t)(b * RB); r < r1; ++r)
                                for (uint32_t p = m.ptr[r]; p < m.ptr[r + 1]; ++p) out[r] += m.val[p];
                        });
                    };
                    row_sums(full.c, rdiag);
                    row_sums(full.ct, cdiag);
                } else {
                    for (uint64_t i = 0; i < d.n_obs; ++i) {
                        double wi = w ? w[i] : 1.0;
                        double lr = kr < 0 ? 1.0 : d.loads[kr][i];
                        double lc = kc < 0 ? 1.0 : d.loads[kc][i];
                        rdiag[rmap[rl[i]]] += wi * lr * lr;
                        cdiag[cmap[cl[i]]] += wi * lc * lc;
                    }
                }
            } else {
            std::vector<uint32_t> cnt(nr + 1, 0);
            for (uint64_t i = 0; i < d.n_obs; ++i) ++cnt[rmap[rl[i]] + 1];
            for (uint32_t i = 0; i < nr; ++i) cnt[i + 1] += cnt[i];
            std::vector<uint32_t> bc(d.n_obs), cur(cnt.begin(), cnt.end() - 1);
            std::vector<double> bv(d.n_obs);
            for (uint64_t i = 0; i < d.n_obs; ++i) {
                uint32_t cj = rmap[rl[i]], ck = cmap[cl[i]];
                double wi = w ? w[i] : 1.0;
                double lr = kr < 0 ? 1.0 : d.loads[kr][i];
                double lc = kc < 0 ? 1.0 : d.loads[kc][i];
                rdiag[cj] += wi * lr * lr;
                cdiag[ck] += wi * lc * lc;
                uint32_t p = cur[cj]++;
                bc[p] = ck;
                bv[p] = wi * lr * lc;
            }
            {
                std::vector<double> work(nc, 0.0);
                std::vector<uint32_t> touched;
                std::vector<char> mark(nc, 0);
                for (uint32_t r = 0; r < nr; ++r) {
                    for (uint32_t p = cnt[r]; p < cnt[r + 1]; ++p) {
                        if (!mark[bc[p]]) { mark[bc[p]] = 1; touched.push_back(bc[p]); }
                        work[bc[p]] += bv[p];
                    }
                    std::sort(touched.begin(), touched.end());
                    for (uint32_t col : touched) {
                        if (work[col] != 0.0) { full.c.col.push_back(col); full.c.val.push_back(work[col]); }
                        work[col] = 0.0;
                        mark[col] = 0;
                    }
                    full.c.ptr.push_back((uint32_t)full.c.col.size());
                    touched.clear();
                }
            }
            std::vector<uint32_t>().swap(bc);
            std::vector<double>().swap(bv);
            full.ct = transpose(full.c);
            }
            if (BuildTrace::on())
                fprintf(stderr, "[within trace]     pair %zu cross-tab %u x %u, %u cells%s\n", pi, nr, nc,
                        full.c.nnz(), cross_tabs ? " (GPU)" : "");
            pst.mark(2);
            const bool known = kr < 0 && kc < 0;
            // components (cross_tab.rs:175-211): label by DFS, then group;
            // numbered in the order of their smallest vertex
            const uint32_t nl = nr + nc;
            std::vector<uint32_t> lab(nl, UINT32_MAX), stk;
            uint32_t ncomp = 0;
            if (cross_tabs && !(*cross_tabs)[pi].comp.empty()) {
                // the GPU's labels (smallest raw vertex of each component; the
                // renumbering of active levels keeps their order, rows before
                // columns), numbered in the same order as the DFS below
                const std::vector<uint32_t>& cm = (*cross_tabs)[pi].comp;
                std::vector<uint32_t> id(cm.size(), UINT32_MAX);
                uint32_t v = 0;
                for (uint32_t j = 0; j < TR.n_levels; ++j)
                    if (active[R.term][j]) {
                        uint32_t& c = id[cm[j]];
                        if (c == UINT32_MAX) c = ncomp++;
                        lab[v++] = c;
                    }
                for (uint32_t k = 0; k < TC.n_levels; ++k)
                    if (active[Cc.term][k]) {
                        uint32_t& c = id[cm[TR.n_levels + k]];
                        if (c == UINT32_MAX) c = ncomp++;
                        lab[v++] = c;
                    }
            }
            for (uint32_t s0 = 0; s0 < nl; ++s0) {
                if (lab[s0] != UINT32_MAX) continue;
                lab[s0] = ncomp;
                stk.push_back(s0);
                while (!stk.empty()) {
                    uint32_t v = stk.back();
                    stk.pop_back();
                    full.nb(v, [&](uint32_t j, double) {
                        if (lab[j] == UINT32_MAX) { lab[j] = ncomp; stk.push_back(j); }
                    });
                }
                ++ncomp;
            }
            pst.mark(3);
            if (BuildTrace::on())
                fprintf(stderr, "[within trace]     pair %zu: %u components after %.3f ms\n", pi, ncomp,
                        (BuildTrace::now() - tr_pair.t0) * 1e3);
            static const char* const steps[] = {"extract", "forms", "lists", "rows", "transpose"};
            StepTimes st(ncomp > 1 ? "components" : "component", steps, 5);
            std::vector<std::vector<uint32_t>> crow(ncomp), ccol(ncomp);
            for (uint32_t i = 0; i < nr; ++i) crow[lab[i]].push_back(i);
            for (uint32_t k = 0; k < nc; ++k) ccol[lab[nr + k]].push_back(k);
            std::vector<uint32_t> rre(nr, UINT32_MAX), cre(nc, UINT32_MAX);
            st.mark(2);
            for (uint32_t ci = 0; ci < ncomp; ++ci) {
                Comp cp;
                std::vector<double> diag;
                if (ncomp == 1) {
                    cp.m = std::move(full);   // the only component: full is not read again
                    diag = rdiag;
                    diag.insert(diag.end(), cdiag.begin(), cdiag.end());
                } else {
                    for (uint32_t i = 0; i < crow[ci].size(); ++i) rre[crow[ci][i]] = i;
                    for (uint32_t i = 0; i < ccol[ci].size(); ++i) cre[ccol[ci][i]] = i;
                    cp.m.c.nr = (uint32_t)crow[ci].size();
                    cp.m.c.nc = (uint32_t)ccol[ci].size();
                    const std::vector<uint32_t>& rows = crow[ci];
                    if (rows.size() >= 65536) {   // rows counted, then filled, by blocks on the host pool
                        const size_t RB = 16384, nb = (rows.size() + RB - 1) / RB;
                        std::vector<uint32_t>& ptr = cp.m.c.ptr;
                        ptr.assign(rows.size() + 1, 0);
                        par_for_each(nb, [&](size_t b) {
                            const size_t i1 = std::min(rows.size(), (b + 1) * RB);
                            for (size_t i = b * RB; i < i1; ++i) {
                                uint32_t c = 0;
                                for (uint32_t k = full.c.ptr[rows[i]]; k < full.c.ptr[rows[i] + 1]; ++k)
                                    c += cre[full.c.col[k]] != UINT32_MAX;
                                ptr[i + 1] = c;
                            }
                        });
                        for (size_t i = 0; i < rows.size(); ++i) ptr[i + 1] += ptr[i];
                        cp.m.c.col.resize(ptr.back());
                        cp.m.c.val.resize(ptr.back());
                        par_for_each(nb, [&](size_t b) {
                            const size_t i1 = std::min(rows.size(), (b + 1) * RB);
                            for (size_t i = b * RB; i < i1; ++i) {
                                uint32_t q = ptr[i];
                                for (uint32_t k = full.c.ptr[rows[i]]; k < full.c.ptr[rows[i] + 1]; ++k) {
                                    const uint32_t nj = cre[full.c.col[k]];
                                    if (nj != UINT32_MAX) {
                                        cp.m.c.col[q] = nj;
                                        cp.m.c.val[q] = full.c.val[k];
                                        ++q;
                                    }
                                }
                            }
                        });
                    } else {
                        for (uint32_t o : rows) {
                            for (uint32_t k = full.c.ptr[o]; k < full.c.ptr[o + 1]; ++k) {
                                uint32_t nj = cre[full.c.col[k]];
                                if (nj != UINT32_MAX) { cp.m.c.col.push_back(nj); cp.m.c.val.push_back(full.c.val[k]); }
                            }
                            cp.m.c.ptr.push_back((uint32_t)cp.m.c.col.size());
                        }
                    }
                    st.mark(3);
                    cp.m.ct = transpose(cp.m.c);
                    st.mark(4);
                    for (uint32_t o : crow[ci]) { rre[o] = UINT32_MAX; diag.push_back(rdiag[o]); }
                    for (uint32_t o : ccol[ci]) { cre[o] = UINT32_MAX; diag.push_back(cdiag[o]); }
                }
                st.mark(0);
                bool allzero = true;
                for (double v : diag) allzero = allzero && v == 0.0;
                if (allzero) {
                    st.mark(1);
                    continue;
                }
                std::vector<uint32_t> globals;
                globals.reserve(crow[ci].size() + ccol[ci].size());
                for (uint32_t o : crow[ci]) globals.push_back(l2g[o]);
                for (uint32_t o : ccol[ci]) globals.push_back(l2g[nr + o]);
                if (cp.m.nc() > cp.m.nr()) {  // orient_for_elimination (sddm.rs:85-106)
                    uint32_t k = cp.m.nr();
                    std::rotate(diag.begin(), diag.begin() + k, diag.end());
                    std::rotate(globals.begin(), globals.begin() + k, globals.end());
                    std::swap(cp.m.c, cp.m.ct);
                }
                bool ok = true, warn = false;
                if (known) {  // convert_known_laplacian (sddm.rs:172-195)
                    auto rs = sums(cp.m, false);
                    double td = 0, tm = 0;
                    for (size_t i = 0; i < diag.size(); ++i) { td += diag[i]; tm += std::fabs(diag[i] - rs[i]); }
                    ok = tm <= budget(64.0, cp.m.nl(), td);
                    cp.diag = rs;
                    cp.ground.assign(cp.m.nl(), 0.0);
                    cp.grounded = false;
                    cp.laplacian = true;
                } else {
                    ok = convert_general(cp, diag, cfg, warn);
                }
                if (!ok) throw WError(ERR_UNSCALABLE, "signed component between term " + std::to_string(R.term) +
                                                          " column " + std::to_string(R.col) + " and term " +
                                                          std::to_string(Cc.term) + " column " + std::to_string(Cc.col) +
                                                          " is not diagonally scalable to SDDM form");
                if (warn) ++n_warnings;
                Domain dm;
                dm.globals = std::move(globals);
                dm.comp = std::move(cp);
                doms.push_back(std::move(dm));
                st.mark(1);
            }
        });
    tr_pairs.done();
    std::vector<Domain> doms;
    for (size_t pi = 0; pi < pairs.size(); ++pi) {
        for (auto& dm : pair_doms[pi]) doms.push_back(std::move(dm));
        out.n_warnings += pair_warnings[pi];
    }
    if (doms.empty()) return out;  // no subdomains: unpreconditioned (operator/schwarz.rs:249-252)

    if (!any_slope) {  // compute_partition_weights (factor_pairs.rs:154-194)
        std::vector<uint32_t> cnt(d.n_dofs, 0);
        for (auto& dm : doms)
            for (uint32_t g : dm.globals) ++cnt[g];
        for (auto& dm : doms) {
            bool uniq = true;
            for (uint32_t g : dm.globals) uniq = uniq && cnt[g] <= 1;
            if (uniq) continue;
            dm.pw.resize(dm.globals.size());
            for (size_t i = 0; i < dm.globals.size(); ++i) dm.pw[i] = 1.0 / std::sqrt((double)cnt[dm.globals[i]]);
        }
    }

    // ---- local solvers: reduced systems and their factors (one domain per host thread) ----
    BuildTrace tr_local("local solvers: reduced systems and factors");
    par_for_each(doms.size(), [&](size_t di) {
        Domain& dm = doms[di];
        const double t_dom = BuildTrace::on() ? BuildTrace::now() : 0.0;
        dm.inv_e = inv_elim(dm.comp);
        if (dm.comp.laplacian) {
            Lap L = reduced_for(dm.comp, dm.inv_e, cfg);
            const double t_red = BuildTrace::on() ? BuildTrace::now() : 0.0;
            factor_lap(L, cfg, dm.fac);
            if (BuildTrace::on() && BuildTrace::now() - t_dom > 0.01)
                fprintf(stderr, "[within trace]     domain %zu reduced system %.3f ms, factor %.3f ms\n", di,
                        (t_red - t_dom) * 1e3, (BuildTrace::now() - t_red) * 1e3);
            dm.mode = dm.comp.grounded ? 1 : 0;
        } else {
            Comp cov = cover_of(dm.comp);
            std::vector<double> inv_c = inv_elim(cov);
            Lap L = reduced_for(cov, inv_c, cfg);
            factor_lap(L, cfg, dm.fac);
            dm.mode = 2;
        }
        if (BuildTrace::on() && BuildTrace::now() - t_dom > 0.01)
            fprintf(stderr, "[within trace]     domain %zu (%u + %u vertices, %u cells) %.3f ms\n", di,
                    dm.comp.m.nr(), dm.comp.m.nc(), dm.comp.m.c.nnz(), (BuildTrace::now() - t_dom) * 1e3);
    });

    tr_local.done();
    BuildTrace tr_pack("pack");
    // ---- pack (layout documented on SchwarzHost) ----
    out.kind = 1;
    SchwarzHost& S = out.schwarz;
    S.n_dofs = (uint32_t)d.n_dofs;
    S.n_sub = (uint32_t)doms.size();
    // per-subdomain offsets into the concatenated arrays (a sequential scan),
    // then every subdomain fills its own ranges on a host thread
    const uint32_t nsub = S.n_sub;
    std::vector<uint64_t> o_loc(nsub + 1, 0), o_el(nsub + 1, 0), o_kp(nsub + 1, 0), o_c(nsub + 1, 0),
        o_ct(nsub + 1, 0), o_red(nsub + 1, 0);
    uint32_t rounds = 0;
    S.loc_ptr.push_back(0);
    S.kept_ptr.push_back(0);
    for (uint32_t s = 0; s < nsub; ++s) {
        const Domain& dm = doms[s];
        o_loc[s + 1] = o_loc[s] + dm.comp.m.nr() + dm.comp.m.nc();
        o_el[s + 1] = o_el[s] + dm.comp.m.nr();
        o_kp[s + 1] = o_kp[s] + dm.comp.m.nc();
        o_c[s + 1] = o_c[s] + dm.comp.m.c.col.size();
        o_ct[s + 1] = o_ct[s] + dm.comp.m.ct.col.size();
        o_red[s + 1] = o_red[s] + dm.fac.n;
        S.n_elim.push_back(dm.comp.m.nr());
        S.n_kept.push_back(dm.comp.m.nc());
        S.red_off.push_back((uint32_t)o_red[s]);
        S.red_n.push_back(dm.fac.n);
        S.mode.push_back(dm.mode);
        S.loc_ptr.push_back((uint32_t)o_loc[s + 1]);
        S.kept_ptr.push_back((uint32_t)o_kp[s + 1]);
        S.cross_nnz += 2ull * dm.comp.m.c.nnz();
        if (!dm.fac.dense) rounds = std::max(rounds, dm.fac.n_rounds);
    }
    const uint32_t red = (uint32_t)o_red[nsub];
    // the arrays (hundreds of MB on large designs) are allocated side by side
    // on host threads: their first-touch page faults and zero fill dominate
    // a sequential allocation
    {
        std::vector<std::function<void()>> allocs = {
            [&] { S.glob.resize(o_loc[nsub]); },       [&] { S.scale.resize(o_loc[nsub]); },
            [&] { S.slot_sub.resize(o_loc[nsub]); },   [&] { S.inv_e.resize(o_loc[nsub]); },
            [&] { S.ct_ptr.resize(o_kp[nsub] + 1); },  [&] { S.ct_rowsum.resize(o_kp[nsub]); },
            [&] { S.ct_row_slot.resize(o_kp[nsub]); }, [&] { S.ct_row_red.resize(o_kp[nsub]); },
            [&] { S.ct_col.resize(o_ct[nsub]); },      [&] { S.ct_val.resize(o_ct[nsub]); },
            [&] { S.c_ptr.resize(o_el[nsub] + 1); },   [&] { S.elim_slot.resize(o_el[nsub]); },
            [&] { S.c_col.resize(o_c[nsub]); },        [&] { S.c_val.resize(o_c[nsub]); },
            [&] { S.red_sub.resize(red); }};
        par_for_each(allocs.size(), [&](size_t i) { allocs[i](); });
    }
    if (BuildTrace::on()) fprintf(stderr, "[within trace]     pack: allocation %.3f ms\n", (BuildTrace::now() - tr_pack.t0) * 1e3);
    // f(lo, hi) over [0, m) in blocks on host threads when m is large (every
    // block writes its own entries, so the result is the sequential loop's)
    auto blocked = [](uint32_t m, auto&& f) {
        constexpr uint32_t BLK = 1u << 16;
        if (m < 4 * BLK) {
            f(0u, m);
            return;
        }
        par_for_each((m + BLK - 1) / BLK, [&](size_t b) {
            const uint32_t lo = (uint32_t)b * BLK;
            f(lo, std::min(m, lo + BLK));
        });
    };
    par_for_each(nsub, [&](size_t si) {
        const uint32_t s = (uint32_t)si;
        const Domain& dm = doms[s];
        const uint32_t ne = dm.comp.m.nr(), nk = dm.comp.m.nc(), nloc = ne + nk;
        const uint32_t lo = (uint32_t)o_loc[s], rd = (uint32_t)o_red[s];
        blocked(nloc, [&](uint32_t j0, uint32_t j1) {
            for (uint32_t j = j0; j < j1; ++j) {
                double f = dm.comp.factors.empty() ? (j < ne ? 1.0 : -1.0) : dm.comp.factors[j];
                double pw = dm.pw.empty() ? 1.0 : dm.pw[j];
                S.glob[lo + j] = dm.globals[j];
                S.scale[lo + j] = pw * f;
                S.slot_sub[lo + j] = s;
                S.inv_e[lo + j] = j < ne ? dm.inv_e[j] : 0.0;
            }
        });
        // C^T rows (kept), columns = local slots of eliminated entries, values
        // pre-divided by D_e (solver.rs:360-371 scales rhs_e by 1/D_e first)
        const Csr& ct = dm.comp.m.ct;
        blocked(nk, [&](uint32_t k0, uint32_t k1) {
            for (uint32_t k = k0; k < k1; ++k) {
                double rs = 0.0;
                for (uint32_t a = ct.ptr[k]; a < ct.ptr[k + 1]; ++a) {
                    const double v = ct.val[a] * dm.inv_e[ct.col[a]];
                    S.ct_col[o_ct[s] + a] = lo + ct.col[a];
                    S.ct_val[o_ct[s] + a] = v;
                    rs += v;
                }
                S.ct_ptr[o_kp[s] + k + 1] = (uint32_t)(o_ct[s] + ct.ptr[k + 1]);
                S.ct_rowsum[o_kp[s] + k] = rs;
                S.ct_row_slot[o_kp[s] + k] = lo + ne + k;
                S.ct_row_red[o_kp[s] + k] = rd + k;
            }
        });
        // C rows (eliminated), columns = reduced slot of the kept entry (bit 31:
        // gauge/cover read-back needed), values pre-divided by D_e (solver.rs:41-77)
        const uint32_t flag = dm.mode == 0 ? 0u : 0x80000000u;
        const Csr& c = dm.comp.m.c;
        blocked(ne, [&](uint32_t e0, uint32_t e1) {
            for (uint32_t e = e0; e < e1; ++e) {
                for (uint32_t a = c.ptr[e]; a < c.ptr[e + 1]; ++a) {
                    S.c_col[o_c[s] + a] = (rd + c.col[a]) | flag;
                    S.c_val[o_c[s] + a] = c.val[a] * dm.inv_e[e];
                }
                S.c_ptr[o_el[s] + e + 1] = (uint32_t)(o_c[s] + c.ptr[e + 1]);
                S.elim_slot[o_el[s] + e] = lo + e;
            }
        });
        for (uint32_t i = 0; i < dm.fac.n; ++i) S.red_sub[rd + i] = s;
    });
    S.n_red = red;
    S.dinv.assign(red, 0.0);
    if (BuildTrace::on()) fprintf(stderr, "[within trace]     pack: slots and C / C^T %.3f ms\n", (BuildTrace::now() - tr_pack.t0) * 1e3);
    // dense blocks
    S.dense_rows_ptr.push_back(0);
    for (uint32_t s = 0; s < S.n_sub; ++s) {
        const Factor& f = doms[s].fac;
        if (!f.dense) continue;
        for (uint32_t r = 0; r < f.n; ++r) {
            for (uint32_t c = 0; c < f.n; ++c) {
                S.dense_col.push_back(S.red_off[s] + c);
                S.dense_val.push_back(f.pinv[(size_t)r * f.n + c]);
            }
            S.dense_rows_ptr.push_back((uint32_t)S.dense_col.size());
            S.dense_row_slot.push_back(S.red_off[s] + r);
        }
        S.factor_nnz += (uint64_t)f.n * f.n;
    }
    // dense cores of round-scheduled factors: x_core = G_core y_core
    S.core_rows_ptr.push_back(0);
    for (uint32_t s = 0; s < S.n_sub; ++s) {
        const Factor& f = doms[s].fac;
        if (f.dense || !f.core_dense) continue;
        const uint32_t m = (uint32_t)f.core.size(), ro = S.red_off[s];
        for (uint32_t i = 0; i < m; ++i) {
            for (uint32_t j = 0; j < m; ++j) {
                S.core_col.push_back(ro + f.core[j]);
                S.core_val.push_back(f.core_pinv[(size_t)i * m + j]);
            }
            S.core_rows_ptr.push_back((uint32_t)S.core_col.size());
            S.core_row_slot.push_back(ro + f.core[i]);
        }
        S.factor_nnz += (uint64_t)m * m;
        S.max_core = std::max(S.max_core, m);
    }
    for (uint32_t s = 0; s < S.n_sub; ++s)
        if (!doms[s].fac.dense) S.max_core = std::max<uint32_t>(S.max_core, (uint32_t)doms[s].fac.core.size());
    // round-scheduled factors: forward rows pull from earlier columns, backward
    // rows (= eliminated columns) pull from later rows.
    S.n_rounds = rounds;
    std::vector<std::vector<uint32_t>> by_round(rounds);
    // rows of each subdomain's L (the transpose of its columns colv), one flat
    // CSR per subdomain: row u lists (reduced slot of column v, l) in ascending v
    struct Rows {
        std::vector<uint32_t> ptr, col;
        std::vector<double> val;
    };
    std::vector<Rows> rowents(S.n_sub);
    par_for_each(S.n_sub, [&](size_t si) {
        const Factor& f = doms[si].fac;
        if (f.dense) return;
        const uint32_t ro = S.red_off[si];
        Rows& R = rowents[si];
        R.ptr.assign((size_t)f.n + 1, 0);
        for (uint32_t v = 0; v < f.n; ++v)
            for (auto& e : f.colv[v]) ++R.ptr[e.first + 1];
        for (uint32_t u = 0; u < f.n; ++u) R.ptr[u + 1] += R.ptr[u];
        R.col.resize(R.ptr[f.n]);
        R.val.resize(R.ptr[f.n]);
        std::vector<uint32_t> cur(R.ptr.begin(), R.ptr.end() - 1);
        for (uint32_t v = 0; v < f.n; ++v)
            for (auto& e : f.colv[v]) {
                const uint32_t q = cur[e.first]++;
                R.col[q] = ro + v;
                R.val[q] = e.second;
            }
    });
    for (uint32_t s = 0; s < S.n_sub; ++s) {
        const Factor& f = doms[s].fac;
        if (f.dense) continue;
        const uint32_t ro = S.red_off[s];
        for (uint32_t v = 0; v < f.n; ++v) {
            S.dinv[ro + v] = f.dinv[v];
            by_round[f.round[v]].push_back(ro + v);
            S.factor_nnz += f.colv[v].size();
        }
    }
    S.fwd_round_ptr.push_back(0);
    S.fwd_ptr.push_back(0);
    S.bwd_round_ptr.push_back(0);
    S.bwd_ptr.push_back(0);
    for (uint32_t r = 0; r < rounds; ++r) {
        S.max_round_rows = std::max<uint32_t>(S.max_round_rows, (uint32_t)by_round[r].size());
        for (uint32_t slot : by_round[r]) {
            uint32_t s = S.red_sub[slot], v = slot - S.red_off[s];
            S.fwd_row.push_back(slot);
            const Rows& R = rowents[s];
            S.fwd_col.insert(S.fwd_col.end(), R.col.begin() + R.ptr[v], R.col.begin() + R.ptr[v + 1]);
            S.fwd_val.insert(S.fwd_val.end(), R.val.begin() + R.ptr[v], R.val.begin() + R.ptr[v + 1]);
            S.fwd_ptr.push_back((uint32_t)S.fwd_col.size());
            S.bwd_row.push_back(slot);
            for (auto& e : doms[s].fac.colv[v]) {
                S.bwd_col.push_back(S.red_off[s] + e.first);
                S.bwd_val.push_back(e.second);
            }
            S.bwd_ptr.push_back((uint32_t)S.bwd_col.size());
        }
        S.fwd_round_ptr.push_back((uint32_t)S.fwd_row.size());
        S.bwd_round_ptr.push_back((uint32_t)S.bwd_row.size());
    }
    if (BuildTrace::on()) fprintf(stderr, "[within trace]     pack: dense blocks and rounds %.3f ms\n", (BuildTrace::now() - tr_pack.t0) * 1e3);
    // prolongation: DOF -> local slots, in subdomain order
    S.dof_ptr.assign(S.n_dofs + 1, 0);
    for (uint32_t g : S.glob) ++S.dof_ptr[g + 1];
    for (uint32_t i = 0; i < S.n_dofs; ++i) S.dof_ptr[i + 1] += S.dof_ptr[i];
    S.dof_slot.resize(S.glob.size());
    {
        std::vector<uint32_t> cur(S.dof_ptr.begin(), S.dof_ptr.end() - 1);
        for (uint32_t j = 0; j < S.glob.size(); ++j) S.dof_slot[cur[S.glob[j]]++] = j;
    }
    return out;
}

// The dense generalised inverse of a symmetric positive semi-definite n x n
// matrix (row-major), as the dense route of the preconditioner builds it;
// empty when a pivot is clearly negative.
std::vector<double> dense_pseudo_inverse(uint32_t n, const std::vector<double>& a) {
    Lap m;
    m.n = n;
    m.ptr.assign(1, 0);
    for (uint32_t i = 0; i < n; ++i) {
        for (uint32_t j = 0; j < n; ++j)
            if (a[(size_t)i * n + j] != 0.0) {
                m.col.push_back(j);
                m.val.push_back(a[(size_t)i * n + j]);
            }
        m.ptr.push_back((uint32_t)m.col.size());
    }
    Factor f;
    if (!dense_pinv(m, f)) return {};
    return f.pinv;
}

}  // namespace wgpu
