// design.cpp -- Design layout, locality sort, operator, slope reparametrisation.
// TEST INFRASTRUCTURE ONLY: CPU FP64 restatement used as the parity checker.
#include "oracle_core.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

namespace orc {

// crates/within/src/domain.rs:110-140 -- stable argsort of observations by a
// level column.  The reference gates a counting sort (n_obs >= n_levels) and a
// stable comparison sort; both yield the same permutation, as here.
void stable_argsort(const uint32_t* key, size_t n_obs, size_t n_levels, uint32_t* perm) {
    if (n_obs < n_levels) {
        for (size_t i = 0; i < n_obs; ++i) perm[i] = (uint32_t)i;
        std::stable_sort(perm, perm + n_obs,
                         [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
        return;
    }
    std::vector<size_t> cursors(n_levels + 1, 0);
    for (size_t i = 0; i < n_obs; ++i) cursors[(size_t)key[i] + 1] += 1;
    for (size_t i = 1; i < cursors.size(); ++i) cursors[i] += cursors[i - 1];
    for (size_t i = 0; i < n_obs; ++i) perm[cursors[key[i]]++] = (uint32_t)i;
}

// crates/within/src/domain/effect.rs:12-42 (validation) and domain.rs:155-247
// (Design::new / Design::build): term-major layout offset_t + c*L_t + level,
// n_levels = max+1, locality sort by the dominant term (the LAST term holding
// the most DOFs, Rust's max_by_key tie rule) when it is not already sorted.
Design build_design(size_t n_obs, size_t n_terms, const uint32_t* codes, const int* intercept,
                    const size_t* n_slopes, const size_t* slope_idx, size_t n_slope_cols,
                    const double* slopes) {
    Design d;
    size_t si = 0;
    for (size_t t = 0; t < n_terms; ++t) {
        TermMeta m;
        if (intercept[t]) m.columns.push_back(-1);
        for (size_t s = 0; s < n_slopes[t]; ++s, ++si) {
            size_t col = slope_idx[si];
            if (col >= n_slope_cols) throw Error(E_BUILD, "slope column index out of range");
            const double* z = slopes + col * n_obs;
            for (size_t i = 0; i < n_obs; ++i)
                if (!std::isfinite(z[i]))
                    throw Error(E_BUILD, "slope " + std::to_string(s) + " loading at index " +
                                             std::to_string(i) + " must be finite");
            d.loads.emplace_back(z, z + n_obs);
            m.columns.push_back((int)d.loads.size() - 1);
        }
        if (m.columns.empty())
            throw Error(E_BUILD, "an effect must have an intercept or at least one slope");
        d.terms.push_back(m);
        d.codes.emplace_back(codes + t * n_obs, codes + (t + 1) * n_obs);
    }
    if (n_obs == 0) throw Error(E_BUILD, "no observations provided");
    d.n_obs = n_obs;
    size_t offset = 0;
    for (size_t q = 0; q < n_terms; ++q) {
        const auto& col = d.codes[q];
        uint32_t mx = 0, prev = 0;
        bool sorted = true;
        for (uint32_t v : col) {
            mx = std::max(mx, v);
            sorted = sorted && v >= prev;
            prev = v;
        }
        auto& m = d.terms[q];
        m.n_levels = (size_t)mx + 1;
        m.offset = offset;
        m.sorted = sorted;
        offset += m.n_dofs();
    }
    if (offset > (size_t)std::numeric_limits<uint32_t>::max())
        throw Error(E_BUILD, "design has " + std::to_string(offset) +
                                 " degrees of freedom, exceeding the u32 column-index limit");
    d.n_dofs = offset;
    if (n_terms > 0) {
        size_t dom = 0;
        for (size_t q = 1; q < n_terms; ++q)
            if (d.terms[q].n_dofs() >= d.terms[dom].n_dofs()) dom = q;
        if (!d.terms[dom].sorted && n_obs <= (size_t)std::numeric_limits<uint32_t>::max()) {
            d.obs_perm.resize(n_obs);
            stable_argsort(d.codes[dom].data(), n_obs, d.terms[dom].n_levels, d.obs_perm.data());
            for (auto& col : d.codes) {
                std::vector<uint32_t> out(n_obs);
                for (size_t i = 0; i < n_obs; ++i) out[i] = col[d.obs_perm[i]];
                col.swap(out);
            }
            for (auto& col : d.loads) {
                std::vector<double> out(n_obs);
                for (size_t i = 0; i < n_obs; ++i) out[i] = col[d.obs_perm[i]];
                col.swap(out);
            }
            for (size_t q = 0; q < n_terms; ++q)
                d.terms[q].sorted = std::is_sorted(d.codes[q].begin(), d.codes[q].end());
        }
    }
    return d;
}

// crates/within/src/operator/design/gather.rs:10-109 -- dst[i] = scale[i] *
// sum_t sum_c src[off_t + c L_t + code_t[i]] * load_c(i); each term's row sum
// folds from -0.0 before it is added to dst (gather.rs:106-107).
void gather_apply(const Design& d, const double* src, double* dst, const double* scale) {
    const size_t n = d.n_obs;
    for (size_t i = 0; i < n; ++i) dst[i] = 0.0;
    for (size_t q = 0; q < d.terms.size(); ++q) {
        const auto& t = d.terms[q];
        const uint32_t* lv = d.codes[q].data();
        par_ranges(n, 65536, [&](size_t a, size_t b, int) {
            for (size_t i = a; i < b; ++i) {
                size_t lev = lv[i];
                double acc = -0.0;
                for (size_t c = 0; c < t.columns.size(); ++c) {
                    double coef = src[t.offset + c * t.n_levels + lev];
                    int k = t.columns[c];
                    acc += (k < 0) ? coef * 1.0 : coef * d.loads[k][i];
                }
                dst[i] += acc;
            }
        });
    }
    if (scale)
        for (size_t i = 0; i < n; ++i) dst[i] *= scale[i];
}

// crates/within/src/operator/design/scatter.rs:14-73 -- the adjoint
// dst[off_t + c L_t + code_t[i]] += load_c(i) * base(i), base = sqrt_w * u.
// The sequential strategy's summation order (observation order) is the
// single-thread reference order.
void scatter_apply(const Design& d, const double* u, const double* sqrt_w, double* dst) {
    const size_t n = d.n_obs;
    for (size_t j = 0; j < d.n_dofs; ++j) dst[j] = 0.0;
    if (g_threads > 1 && n >= 65536) {   // timing mode: per-thread accumulators summed in thread order
        const int T = g_threads;
        std::vector<double> part((size_t)T * d.n_dofs, 0.0);
        par_ranges(n, 0, [&](size_t a, size_t b, int tid) {
            double* my = part.data() + (size_t)tid * d.n_dofs;
            for (size_t i = a; i < b; ++i) {
                double bv = sqrt_w ? sqrt_w[i] * u[i] : u[i];
                for (size_t q = 0; q < d.terms.size(); ++q) {
                    const auto& t = d.terms[q];
                    const uint32_t lv = d.codes[q][i];
                    for (size_t c = 0; c < t.columns.size(); ++c) {
                        int k = t.columns[c];
                        my[t.offset + c * t.n_levels + lv] += (k < 0) ? bv : d.loads[k][i] * bv;
                    }
                }
            }
        });
        par_ranges(d.n_dofs, 0, [&](size_t a, size_t b, int) {
            for (size_t j = a; j < b; ++j) {
                double s = 0.0;
                for (int r = 0; r < T; ++r) s += part[(size_t)r * d.n_dofs + j];
                dst[j] = s;
            }
        });
        return;
    }
    for (size_t q = 0; q < d.terms.size(); ++q) {
        const auto& t = d.terms[q];
        const uint32_t* lv = d.codes[q].data();
        for (size_t i = 0; i < n; ++i) {
            double b = sqrt_w ? sqrt_w[i] * u[i] : u[i];
            for (size_t c = 0; c < t.columns.size(); ++c) {
                int k = t.columns[c];
                double v = (k < 0) ? b : d.loads[k][i] * b;
                dst[t.offset + c * t.n_levels + lv[i]] += v;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// crates/within/src/solver/reparam.rs -- per-level whitening of slope columns.

static const double RANK_TOL = 1e-10;  // reparam.rs:13

static inline size_t tri_index(size_t j, size_t k) { return j * (j + 1) / 2 + k; }
static inline size_t tri_len(size_t v) { return v * (v + 1) / 2; }
static double dotv(const double* a, const double* b, size_t n) {
    double s = 0;
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

// reparam.rs:284-316 -- pivoted Gram-Schmidt in coordinates of the level Gram.
static void pivoted_gram_schmidt(const std::vector<double>& g, size_t v, double tol,
                                 std::vector<double>& basis, std::vector<bool>& kept) {
    std::vector<double> residual(v);
    for (size_t j = 0; j < v; ++j) residual[j] = g[j * v + j];
    kept.assign(v, false);
    basis.clear();
    for (;;) {
        // max_by over total_cmp returns the last maximal element.
        long p = -1;
        for (size_t j = 0; j < v; ++j) {
            if (kept[j] || !std::isfinite(residual[j]) || !(residual[j] > tol * g[j * v + j]))
                continue;
            if (p < 0 || !(residual[j] < residual[p])) p = (long)j;
        }
        if (p < 0) break;
        kept[p] = true;
        std::vector<double> q(v, 0.0);
        q[p] = 1.0;
        for (size_t b = 0; b + v <= basis.size(); b += v) {
            double c = dotv(&g[p * v], &basis[b], v);
            for (size_t j = 0; j < v; ++j) q[j] -= c * basis[b + j];
        }
        double norm = std::sqrt(residual[p]);
        for (auto& qj : q) qj /= norm;
        for (size_t j = 0; j < v; ++j) {
            double c = dotv(&g[j * v], q.data(), v);
            residual[j] -= c * c;
        }
        basis.insert(basis.end(), q.begin(), q.end());
    }
}

SlopeReparam build_reparam(Design& d, const double* weights) {
    SlopeReparam out;
    for (size_t term = 0; term < d.terms.size(); ++term) {
        const TermMeta& meta = d.terms[term];
        bool any = false;
        for (int c : meta.columns) any = any || c >= 0;
        if (!any) continue;
        TermReparam tr;
        tr.offset = meta.offset;
        tr.n_levels = meta.n_levels;
        std::vector<size_t> z_cols;
        for (size_t c = 0; c < meta.columns.size(); ++c) {
            if (meta.columns[c] >= 0) {
                tr.slope_columns.push_back(c);
                z_cols.push_back((size_t)meta.columns[c]);
            } else {
                tr.intercept_column = (int)c;
            }
        }
        const bool intercept = tr.intercept_column >= 0;
        const size_t v = z_cols.size();
        const size_t L = meta.n_levels;
        const uint32_t* levels = d.codes[term].data();
        // LevelMoments (reparam.rs:203-276): weighted multivariate Welford.
        std::vector<double> w_sum(L, 0.0), mean(L * v, 0.0), com(L * tri_len(v), 0.0), delta(v);
        std::vector<double> z_row(v);
        for (size_t i = 0; i < d.n_obs; ++i) {
            for (size_t j = 0; j < v; ++j) z_row[j] = d.loads[z_cols[j]][i];
            double w = weights ? weights[i] : 1.0;
            if (w <= 0.0) continue;
            size_t lev = levels[i];
            w_sum[lev] += w;
            double ratio = w / w_sum[lev];
            double* mu = &mean[lev * v];
            for (size_t j = 0; j < v; ++j) {
                delta[j] = z_row[j] - mu[j];
                mu[j] += ratio * delta[j];
            }
            double* cm = &com[lev * tri_len(v)];
            for (size_t j = 0; j < v; ++j) {
                double dev = w * (z_row[j] - mu[j]);
                for (size_t k = 0; k <= j; ++k) cm[tri_index(j, k)] += delta[k] * dev;
            }
        }
        std::vector<double> gram(v * v), basis;
        std::vector<bool> kept;
        tr.transforms.resize(L);
        for (size_t level = 0; level < L; ++level) {
            const double* cm = &com[level * tri_len(v)];
            const double* mu = &mean[level * v];
            for (size_t j = 0; j < v; ++j)
                for (size_t k = 0; k <= j; ++k) {
                    double g = cm[tri_index(j, k)];
                    if (!intercept) g += w_sum[level] * mu[j] * mu[k];
                    gram[j * v + k] = g;
                    gram[k * v + j] = g;
                }
            pivoted_gram_schmidt(gram, v, RANK_TOL, basis, kept);
            if (intercept && w_sum[level] == 0.0)
                out.unidentified.push_back({term, level, 0});
            for (size_t j = 0; j < v; ++j)
                if (!kept[j]) out.unidentified.push_back({term, level, tr.slope_columns[j]});
            tr.transforms[level].w = basis;
            if (intercept)
                tr.transforms[level].center.assign(mu, mu + v);
            else
                tr.transforms[level].center.assign(v, 0.0);
        }
        std::vector<std::vector<double>> u_cols(v, std::vector<double>(d.n_obs, 0.0));
        for (size_t i = 0; i < d.n_obs; ++i) {
            const auto& t = tr.transforms[levels[i]];
            for (size_t j = 0; j < v; ++j) z_row[j] = d.loads[z_cols[j]][i] - t.center[j];
            for (size_t r = 0; r * v < t.w.size(); ++r)
                u_cols[r][i] = dotv(&t.w[r * v], z_row.data(), v);
        }
        for (size_t j = 0; j < v; ++j) d.loads[z_cols[j]].swap(u_cols[j]);
        out.terms.push_back(std::move(tr));
    }
    out.active = !out.terms.empty();
    return out;
}

// reparam.rs:173-194
void TermReparam::back_transform(double* x) const {
    const size_t v = slope_columns.size();
    std::vector<double> b(v);
    for (size_t l = 0; l < transforms.size(); ++l) {
        const auto& t = transforms[l];
        if (t.w.empty()) continue;
        std::fill(b.begin(), b.end(), 0.0);
        for (size_t k = 0; k * v < t.w.size(); ++k) {
            double bk = x[offset + slope_columns[k] * n_levels + l];
            for (size_t j = 0; j < v; ++j) b[j] += t.w[k * v + j] * bk;
        }
        for (size_t j = 0; j < v; ++j) x[offset + slope_columns[j] * n_levels + l] = b[j];
        if (intercept_column >= 0)
            x[offset + (size_t)intercept_column * n_levels + l] -= dotv(b.data(), t.center.data(), v);
    }
}

}  // namespace orc
