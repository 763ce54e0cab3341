// host_design.cpp -- design lowering, locality sort, slope reparametrisation
// and segmented-reduction tile plans (host side, once per Solver).
#include <algorithm>
#include <cmath>
#include <limits>
#include <memory>
#include <numeric>

#include "host.hpp"
#include "host_pool.hpp"

namespace wgpu {

// Stable argsort of observations by level (crates/within/src/domain.rs:110-140).
// The reference switches between a counting sort and a stable comparison sort
// on n_obs < n_levels; both give the same permutation, which is all that is
// observable, so the counting sort runs whenever its bucket array is small.
//
// A large input is sorted in two stable passes on the host pool: chunks of
// the input partition the indices by the key's top 11 bits (per-chunk counts,
// so every bucket keeps input order), then every bucket is counting-sorted by
// the full key on its own; equal keys share a bucket and keep their order, so
// the result is the same stable permutation.
void stable_argsort_u32(const uint32_t* key, size_t n, size_t n_levels, uint32_t* perm) {
    if (n < n_levels && n_levels > (size_t)1 << 26) {
        for (size_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
        std::stable_sort(perm, perm + n, [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
        return;
    }
    if (n >= ((size_t)1 << 20) && n_levels <= ((size_t)1 << 26)) {
        int bits = 0;
        while (((size_t)1 << bits) < n_levels) ++bits;
        const int hb = std::min(bits, 11), shift = bits - hb;
        const size_t NB = (size_t)1 << hb, nch = 16, per = (n + nch - 1) / nch;
        std::vector<size_t> cnt(nch * NB, 0);
        par_for_each(nch, [&](size_t t) {
            size_t* c = &cnt[t * NB];
            const size_t i1 = std::min(n, (t + 1) * per);
            for (size_t i = t * per; i < i1; ++i) ++c[key[i] >> shift];
        });
        std::vector<size_t> bstart(NB + 1, 0);
        size_t o = 0;
        for (size_t b = 0; b < NB; ++b) {
            bstart[b] = o;
            for (size_t t = 0; t < nch; ++t) {
                const size_t c = cnt[t * NB + b];
                cnt[t * NB + b] = o;
                o += c;
            }
        }
        bstart[NB] = o;
        // with at most 2^11 levels the partition is the whole sort
        std::unique_ptr<uint32_t[]> tmp(shift ? new uint32_t[n] : nullptr);   // first touched by the scatter
        uint32_t* dst = shift ? tmp.get() : perm;
        par_for_each(nch, [&](size_t t) {
            size_t* c = &cnt[t * NB];
            const size_t i1 = std::min(n, (t + 1) * per);
            for (size_t i = t * per; i < i1; ++i) dst[c[key[i] >> shift]++] = (uint32_t)i;
        });
        if (!shift) return;
        const size_t width = (size_t)1 << shift, BB = 16;
        par_for_each((NB + BB - 1) / BB, [&](size_t g) {
            std::vector<uint32_t> h(width + 1);
            for (size_t b = g * BB; b < std::min(NB, (g + 1) * BB); ++b) {
                const size_t b0 = bstart[b], b1 = bstart[b + 1];
                if (b0 == b1) continue;
                std::fill(h.begin(), h.end(), 0u);
                const uint32_t base = (uint32_t)(b << shift);
                for (size_t q = b0; q < b1; ++q) ++h[key[tmp[q]] - base + 1];
                for (size_t l = 0; l < width; ++l) h[l + 1] += h[l];
                for (size_t q = b0; q < b1; ++q) perm[b0 + h[key[tmp[q]] - base]++] = tmp[q];
            }
        });
        return;
    }
    std::vector<uint64_t> cur(n_levels + 1, 0);
    for (size_t i = 0; i < n; ++i) ++cur[(size_t)key[i] + 1];
    for (size_t l = 0; l < n_levels; ++l) cur[l + 1] += cur[l];
    for (size_t i = 0; i < n; ++i) perm[cur[key[i]]++] = (uint32_t)i;
}

// Design::new / Design::build (domain.rs:155-247) with Effect::new validation
// (effect.rs:12-42): term-major layout, n_levels = max code + 1, sortedness
// flags, and the locality sort by the dominant term -- the last term holding
// the most DOFs (Rust's max_by_key tie rule), applied when it is unsorted.
HostDesign make_design(uint64_t n_obs, const std::vector<EffectIn>& effects) {
    HostDesign d;
    if (effects.size() > (size_t)MAX_TERMS)
        throw WError(ERR_UNSUPPORTED, "at most " + std::to_string(MAX_TERMS) + " effects are supported");
    // the finiteness of every slope column, checked side by side (the first
    // failing column in effect order is reported, at its first bad index)
    std::vector<const double*> zcols;
    for (const EffectIn& ef : effects)
        for (const double* z : ef.slopes) zcols.push_back(z);
    std::vector<uint64_t> bad(zcols.size(), UINT64_MAX);
    par_for_each(zcols.size(), [&](size_t j) {
        for (uint64_t i = 0; i < n_obs; ++i)
            if (!std::isfinite(zcols[j][i])) {
                bad[j] = i;
                break;
            }
    });
    size_t zj = 0;
    for (size_t e = 0; e < effects.size(); ++e) {
        const EffectIn& ef = effects[e];
        Term t;
        if (ef.intercept) t.cols.push_back(-1);
        for (size_t s = 0; s < ef.slopes.size(); ++s, ++zj) {
            if (bad[zj] != UINT64_MAX)
                throw WError(ERR_BUILD, "slope " + std::to_string(s) + " loading at index " +
                                            std::to_string(bad[zj]) + " must be finite, got " +
                                            std::to_string(ef.slopes[s][bad[zj]]));
            t.cols.push_back((int)zj);
        }
        if (t.cols.empty()) throw WError(ERR_BUILD, "an effect must have an intercept or at least one slope");
        if (t.cols.size() > (size_t)MAX_COLS)
            throw WError(ERR_UNSUPPORTED, "at most " + std::to_string(MAX_COLS - 1) + " slopes per effect are supported");
        d.terms.push_back(t);
    }
    if (zcols.size() > (size_t)MAX_LOADS)
        throw WError(ERR_UNSUPPORTED, "at most " + std::to_string(MAX_LOADS) + " slope columns are supported");
    if (n_obs == 0) throw WError(ERR_BUILD, "no observations provided");
    if (n_obs > (uint64_t)std::numeric_limits<uint32_t>::max())
        throw WError(ERR_UNSUPPORTED, "more than 2^32-1 observations in one design");
    d.n_obs = n_obs;
    // codes and loading columns copied, and every term's largest code and
    // sortedness found, side by side
    d.codes.resize(effects.size());
    d.loads.resize(zcols.size());
    std::vector<uint32_t> mxs(effects.size(), 0);
    std::vector<char> srt(effects.size(), 1);
    par_for_each(effects.size() + zcols.size(), [&](size_t i) {
        if (i < effects.size()) {
            d.codes[i].assign(effects[i].levels, effects[i].levels + n_obs);
            uint32_t mx = 0, prev = 0;
            bool sorted = true;
            for (uint32_t v : d.codes[i]) {
                mx = std::max(mx, v);
                sorted = sorted && v >= prev;
                prev = v;
            }
            mxs[i] = mx;
            srt[i] = sorted ? 1 : 0;
        } else {
            const size_t j = i - effects.size();
            d.loads[j].assign(zcols[j], zcols[j] + n_obs);
        }
    });
    uint64_t offset = 0;
    for (size_t q = 0; q < d.terms.size(); ++q) {
        Term& t = d.terms[q];
        uint64_t nl = (uint64_t)mxs[q] + 1;
        t.sorted = srt[q] != 0;
        t.offset = (uint32_t)std::min<uint64_t>(offset, std::numeric_limits<uint32_t>::max());
        offset += nl * t.cols.size();
        t.n_levels = (uint32_t)std::min<uint64_t>(nl, std::numeric_limits<uint32_t>::max());
    }
    if (offset > (uint64_t)std::numeric_limits<uint32_t>::max())
        throw WError(ERR_BUILD, "design has " + std::to_string(offset) +
                                    " degrees of freedom, exceeding the u32 column-index limit");
    d.n_dofs = offset;
    if (!d.terms.empty()) {
        size_t dom = 0;
        for (size_t q = 1; q < d.terms.size(); ++q)
            if (d.terms[q].n_dofs() >= d.terms[dom].n_dofs()) dom = q;
        if (!d.terms[dom].sorted) {
            d.obs_perm.resize(n_obs);
            stable_argsort_u32(d.codes[dom].data(), n_obs, d.terms[dom].n_levels, d.obs_perm.data());
            // gathers by ranges of observations on the host pool
            const size_t nch = n_obs >= ((uint64_t)1 << 20) ? 16 : 1, per = (n_obs + nch - 1) / nch;
            const uint32_t* pm = d.obs_perm.data();
            std::vector<uint32_t> tmp(n_obs);
            for (auto& col : d.codes) {
                par_for_each(nch, [&](size_t t) {
                    const uint64_t i1 = std::min<uint64_t>(n_obs, (t + 1) * per);
                    for (uint64_t i = t * per; i < i1; ++i) tmp[i] = col[pm[i]];
                });
                col.swap(tmp);
            }
            std::vector<double> tz(n_obs);
            for (auto& col : d.loads) {
                par_for_each(nch, [&](size_t t) {
                    const uint64_t i1 = std::min<uint64_t>(n_obs, (t + 1) * per);
                    for (uint64_t i = t * per; i < i1; ++i) tz[i] = col[pm[i]];
                });
                col.swap(tz);
            }
            for (size_t q = 0; q < d.terms.size(); ++q)
                d.terms[q].sorted = std::is_sorted(d.codes[q].begin(), d.codes[q].end());
        }
    }
    return d;
}

// ---------------------------------------------------------------------------
// Slope reparametrisation (crates/within/src/solver/reparam.rs:48-316): per
// level, weighted Welford moments of the slope covariates, a pivoted
// Gram-Schmidt in the coordinates of the level Gram (RANK_TOL = 1e-10), and
// the loading columns overwritten by the whitened u = W (z - center).

namespace {
constexpr double RANK_TOL = 1e-10;
inline size_t tri(size_t j, size_t k) { return j * (j + 1) / 2 + k; }

void pivoted_gs(const std::vector<double>& g, size_t v, std::vector<double>& basis,
                std::vector<char>& kept) {
    std::vector<double> res(v);
    for (size_t j = 0; j < v; ++j) res[j] = g[j * v + j];
    kept.assign(v, 0);
    basis.clear();
    for (;;) {
        long p = -1;
        for (size_t j = 0; j < v; ++j) {
            if (kept[j] || !std::isfinite(res[j]) || !(res[j] > RANK_TOL * g[j * v + j])) continue;
            if (p < 0 || !(res[j] < res[p])) p = (long)j;
        }
        if (p < 0) return;
        kept[p] = 1;
        std::vector<double> q(v, 0.0);
        q[p] = 1.0;
        for (size_t b = 0; b < basis.size(); b += v) {
            double c = 0;
            for (size_t j = 0; j < v; ++j) c += g[p * v + j] * basis[b + j];
            for (size_t j = 0; j < v; ++j) q[j] -= c * basis[b + j];
        }
        double nrm = std::sqrt(res[p]);
        for (double& x : q) x /= nrm;
        for (size_t j = 0; j < v; ++j) {
            double c = 0;
            for (size_t i = 0; i < v; ++i) c += g[j * v + i] * q[i];
            res[j] -= c * c;
        }
        basis.insert(basis.end(), q.begin(), q.end());
    }
}
}  // namespace

Reparam build_reparam(HostDesign& d, const double* w) {
    Reparam out;
    for (size_t term = 0; term < d.terms.size(); ++term) {
        const Term& t = d.terms[term];
        std::vector<uint32_t> zc;
        Reparam::TermR tr;
        tr.offset = t.offset;
        tr.n_levels = t.n_levels;
        for (size_t c = 0; c < t.cols.size(); ++c) {
            if (t.cols[c] < 0) {
                tr.intercept_col = (int)c;
            } else {
                tr.slope_cols.push_back((uint32_t)c);
                zc.push_back((uint32_t)t.cols[c]);
            }
        }
        if (zc.empty()) continue;
        const bool icpt = tr.intercept_col >= 0;
        const size_t v = zc.size(), L = t.n_levels, tl = v * (v + 1) / 2;
        const uint32_t* lev = d.codes[term].data();
        std::vector<double> wsum(L, 0.0), mean(L * v, 0.0), com(L * tl, 0.0), delta(v), z(v);
        for (uint64_t i = 0; i < d.n_obs; ++i) {
            double wi = w ? w[i] : 1.0;
            if (wi <= 0.0) continue;
            size_t l = lev[i];
            for (size_t j = 0; j < v; ++j) z[j] = d.loads[zc[j]][i];
            wsum[l] += wi;
            double ratio = wi / wsum[l];
            double* mu = &mean[l * v];
            for (size_t j = 0; j < v; ++j) {
                delta[j] = z[j] - mu[j];
                mu[j] += ratio * delta[j];
            }
            double* cm = &com[l * tl];
            for (size_t j = 0; j < v; ++j) {
                double dev = wi * (z[j] - mu[j]);
                for (size_t k = 0; k <= j; ++k) cm[tri(j, k)] += delta[k] * dev;
            }
        }
        tr.w.resize(L);
        tr.center.resize(L);
        std::vector<double> g(v * v), basis;
        std::vector<char> kept;
        for (size_t l = 0; l < L; ++l) {
            const double* cm = &com[l * tl];
            const double* mu = &mean[l * v];
            for (size_t j = 0; j < v; ++j)
                for (size_t k = 0; k <= j; ++k) {
                    double gv = cm[tri(j, k)];
                    if (!icpt) gv += wsum[l] * mu[j] * mu[k];
                    g[j * v + k] = gv;
                    g[k * v + j] = gv;
                }
            pivoted_gs(g, v, basis, kept);
            if (icpt && wsum[l] == 0.0) {
                out.unidentified.insert(out.unidentified.end(), {term, l, 0});
            }
            for (size_t j = 0; j < v; ++j)
                if (!kept[j]) out.unidentified.insert(out.unidentified.end(), {term, l, tr.slope_cols[j]});
            tr.w[l] = basis;
            if (icpt) tr.center[l].assign(mu, mu + v);
            else tr.center[l].assign(v, 0.0);
        }
        std::vector<std::vector<double>> u(v, std::vector<double>(d.n_obs, 0.0));
        for (uint64_t i = 0; i < d.n_obs; ++i) {
            size_t l = lev[i];
            const auto& wl = tr.w[l];
            const auto& cl = tr.center[l];
            for (size_t j = 0; j < v; ++j) z[j] = d.loads[zc[j]][i] - cl[j];
            for (size_t r = 0; r * v < wl.size(); ++r) {
                double s = 0;
                for (size_t j = 0; j < v; ++j) s += wl[r * v + j] * z[j];
                u[r][i] = s;
            }
        }
        for (size_t j = 0; j < v; ++j) d.loads[zc[j]].swap(u[j]);
        out.terms.push_back(std::move(tr));
    }
    return out;
}

// reparam.rs:173-194
void Reparam::back_transform(double* x) const {
    for (const auto& t : terms) {
        const size_t v = t.slope_cols.size();
        std::vector<double> b(v);
        for (size_t l = 0; l < t.w.size(); ++l) {
            const auto& wl = t.w[l];
            if (wl.empty()) continue;
            std::fill(b.begin(), b.end(), 0.0);
            for (size_t k = 0; k * v < wl.size(); ++k) {
                double bk = x[t.offset + (size_t)t.slope_cols[k] * t.n_levels + l];
                for (size_t j = 0; j < v; ++j) b[j] += wl[k * v + j] * bk;
            }
            for (size_t j = 0; j < v; ++j) x[t.offset + (size_t)t.slope_cols[j] * t.n_levels + l] = b[j];
            if (t.intercept_col >= 0) {
                double s = 0;
                for (size_t j = 0; j < v; ++j) s += b[j] * t.center[l][j];
                x[t.offset + (size_t)t.intercept_col * t.n_levels + l] -= s;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Tile plan of one segmented-reduction problem (see segreduce.cuh).
void HostPlan::add(uint32_t problem, const uint32_t* ptr, uint32_t n_seg, int T) {
    // Positions of this problem are [ptr[0], ptr[n_seg]).  Tiles hold at most
    // T positions and own at most T segments (a run of empty segments, e.g.
    // the first round of a triangular solve, is spread over several CTAs; a
    // tile may then own segments but no positions).
    const uint32_t pbase = ptr[0], pend = ptr[n_seg];
    const uint32_t base = (uint32_t)tiles.size();
    uint32_t p = pbase, s = 0;
    std::vector<uint32_t> starts;  // p0 of tiles holding positions, for split lookup
    std::vector<uint32_t> ids;
    do {
        SRTile t{};
        t.problem = problem;
        t.p0 = p;
        t.own_lo = s;
        uint32_t hi = (uint32_t)std::min<uint64_t>((uint64_t)p + (uint32_t)T, pend);
        uint32_t owned = 0;
        const bool at_end = p == pend;
        while (s < n_seg && (ptr[s] < hi || (at_end && ptr[s] == pend)) && owned < (uint32_t)T) {
            ++s;
            ++owned;
        }
        if (owned == (uint32_t)T && s < n_seg && ptr[s] < hi) hi = ptr[s];  // segment budget spent
        t.p1 = hi;
        t.own_hi = s;
        t.cont_split = -1;
        t.tail_split = -1;
        if (t.p1 > t.p0) {
            starts.push_back(t.p0);
            ids.push_back((uint32_t)tiles.size());
        }
        tiles.push_back(t);
        p = hi;
    } while (p < pend || s < n_seg);
    // split segments: positions spread over more than one tile.  The tile of
    // a position is the last position-holding tile starting at or before it;
    // segment starts and ends only grow with g, so two cursors find them.
    size_t ca = 0, cb = 0;
    auto tile_of = [&](uint32_t pos, size_t& c) {
        while (c + 1 < starts.size() && starts[c + 1] <= pos) ++c;
        return ids[c];
    };
    for (uint32_t g = 0; g < n_seg; ++g) {
        uint32_t a = ptr[g], b = ptr[g + 1];
        if (b <= a) continue;
        uint32_t t0 = tile_of(a, ca), t1 = tile_of(b - 1, cb);
        if (t1 == t0) continue;
        int id = (int)splits.size();
        splits.push_back(SRSplit{problem, g, t0, t1});
        tiles[t0].tail_split = id;
        for (uint32_t t = t0 + 1; t <= t1; ++t) tiles[t].cont_split = id;
    }
    (void)base;
}

uint32_t ss_range_len(uint64_t positions, uint32_t warps) {
    const uint64_t per = (positions + std::max<uint32_t>(1, warps) - 1) / std::max<uint32_t>(1, warps);
    const uint64_t len = (per + SS_ALIGN - 1) / SS_ALIGN * SS_ALIGN;
    return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(len, SS_ALIGN), 1u << 16);
}

void SSHostPlan::add(uint32_t problem, const uint32_t* ptr, uint32_t n_seg, uint32_t L) {
    if (n_seg == 0) return;
    const uint32_t ptr0 = ptr[0], pend = ptr[n_seg];
    const uint32_t P = pend - ptr0;
    // segment-start bitmap: bit (p - ptr0) is set where a non-empty segment
    // starts; words past the last position cover the reads of a full last
    // chunk (up to 3 words beyond it at 4 positions per lane)
    const uint32_t word0 = (uint32_t)bits.size();
    bits.resize((size_t)word0 + (P + 31) / 32 + 4, 0u);
    std::vector<uint32_t> nz;   // non-empty segment ids in order
    nz.reserve(n_seg);
    bool has_empty = false;
    for (uint32_t g = 0; g < n_seg; ++g) {
        if (ptr[g + 1] > ptr[g]) {
            nz.push_back(g);
            const uint32_t b = ptr[g] - ptr0;
            bits[(size_t)word0 + b / 32] |= 1u << (b % 32);
        } else {
            has_empty = true;
        }
    }
    uint32_t nz_off = SS_IDENTITY;
    if (has_empty) {
        nz_off = (uint32_t)nz_ids.size();
        nz_ids.insert(nz_ids.end(), nz.begin(), nz.end());
    }
    const uint32_t nr = P == 0 ? 1u : (P + L - 1) / L;
    const uint32_t r_first = (uint32_t)ranges.size();
    size_t q = 0;   // nz[q] is the non-empty segment holding the range's first position
    for (uint32_t j = 0; j < nr; ++j) {
        SSRange r{};
        r.problem = problem;
        r.p0 = ptr0 + j * L;
        r.p1 = (uint32_t)std::min<uint64_t>((uint64_t)r.p0 + L, pend);
        r.word0 = word0 + (j * L) / 32;
        while (q + 1 < nz.size() && ptr[nz[q + 1]] <= r.p0) ++q;
        r.o0 = (uint32_t)q;
        r.head_split = -1;
        r.tail_split = -1;
        r.nz_off = nz_off;
        ranges.push_back(r);
    }
    // split segments: positions in more than one range
    for (size_t o = 0; o < nz.size(); ++o) {
        const uint32_t g = nz[o], a = ptr[g] - ptr0, b = ptr[g + 1] - ptr0;
        const uint32_t r0 = a / L, r1 = (b - 1) / L;
        if (r1 == r0) continue;
        const int id = (int)splits.size();
        splits.push_back(SSSplit{problem, g, r_first + r0, r_first + r1});
        ranges[r_first + r0].tail_split = id;
        for (uint32_t t = r0 + 1; t <= r1; ++t) ranges[r_first + t].head_split = id;
    }
    // empty segments go to the range holding their position (the last range
    // for those at the problem's end); the list is in range order
    std::vector<uint32_t> cnt(nr, 0);
    for (uint32_t g = 0; g < n_seg; ++g)
        if (ptr[g + 1] == ptr[g]) {
            const uint32_t rel = ptr[g] - ptr0;
            ++cnt[std::min(nr - 1, rel / L)];
        }
    uint32_t e = (uint32_t)empties.size();
    for (uint32_t j = 0; j < nr; ++j) {
        ranges[r_first + j].e_lo = e;
        e += cnt[j];
        ranges[r_first + j].e_hi = ranges[r_first + j].e_lo;
    }
    empties.resize(e);
    for (uint32_t g = 0; g < n_seg; ++g)
        if (ptr[g + 1] == ptr[g]) {
            const uint32_t rel = ptr[g] - ptr0;
            SSRange& r = ranges[r_first + std::min(nr - 1, rel / L)];
            empties[r.e_hi++] = g;
        }
}

}  // namespace wgpu
