// Property test of the additive-Schwarz host image (build_preconditioner):
//  - the round schedule of the approximate-Cholesky factors, which the apply
//    kernels run one round per launch with every row of a round in parallel:
//    a forward row reads only rows of earlier rounds, and a backward row reads
//    only rows of later rounds (solved earlier on the way back) or rows whose
//    own backward update is empty (core vertices: rewritten unchanged);
//  - the index range of every array the apply kernels gather through.
//  - the host image does not depend on the number of host threads that
//    built it (WITHIN_HOST_THREADS=1 against the default).
// Random worker/firm/year-like designs (every fourth with a slope on the second
// factor and observation weights, which takes the signed / cover routes of the
// set-up), with the round stop rules relaxed so that several rounds are
// scheduled; two large ones run the threaded rounds.
#include "host.hpp"

#include <cstdio>
#include <cstdlib>
#include <random>

using namespace wgpu;

static uint64_t fnv(uint64_t h, const void* p, size_t n) {
    const unsigned char* b = (const unsigned char*)p;
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}
template <class T>
static uint64_t fnv(uint64_t h, const std::vector<T>& v) {
    return v.empty() ? fnv(h, "", 0) : fnv(h, v.data(), v.size() * sizeof(T));
}
static uint64_t image_hash(const SchwarzHost& S) {
    uint64_t h = 1469598103934665603ull;
    h = fnv(h, S.glob); h = fnv(h, S.scale); h = fnv(h, S.inv_e); h = fnv(h, S.mode);
    h = fnv(h, S.ct_ptr); h = fnv(h, S.ct_col); h = fnv(h, S.ct_val); h = fnv(h, S.c_ptr);
    h = fnv(h, S.c_col); h = fnv(h, S.c_val); h = fnv(h, S.dense_val); h = fnv(h, S.dinv);
    h = fnv(h, S.fwd_row); h = fnv(h, S.fwd_col); h = fnv(h, S.fwd_val); h = fnv(h, S.bwd_col);
    h = fnv(h, S.bwd_val); h = fnv(h, S.core_val); h = fnv(h, S.dof_slot);
    return h;
}

static int fail(const char* what, int trial) {
    printf("FAIL %s (trial %d)\n", what, trial);
    return 1;
}

int main() {
    std::mt19937_64 rng(11);
    uint64_t rounds_seen = 0, rows_checked = 0, not_laplacian = 0;
    for (int trial = 0; trial < 26; ++trial) {
        // the last two: a reduced system of ~20,000 vertices, whose rounds run on host threads
        const bool big = trial >= 24;
        const uint32_t n = big ? 160000 : 4000 + (uint32_t)(rng() % 20000);
        const uint32_t L0 = big ? 60000 : 300 + (uint32_t)(rng() % 2000);
        const uint32_t L1 = big ? 20000 : 80 + (uint32_t)(rng() % 400);
        const uint32_t L2 = 3 + (uint32_t)(rng() % 30);
        std::vector<uint32_t> a(n), b(n), c(n);
        std::vector<double> z(n), w(n);
        // clustered first factor (panel-like runs), random others
        uint32_t cur = 0;
        for (uint32_t i = 0; i < n; ++i) {
            if (i < L0) cur = i;
            else if (rng() % 8 == 0) cur = (uint32_t)(rng() % L0);
            a[i] = cur;
            b[i] = i < L1 ? i : (uint32_t)(rng() % L1);
            c[i] = i < L2 ? i : (uint32_t)(rng() % L2);
            z[i] = (double)(rng() % 2001) / 1000.0 - 1.0;
            w[i] = 0.25 + (double)(rng() % 1000) / 500.0;
        }
        const bool slopes = trial % 4 == 3;
        std::vector<EffectIn> eff;
        eff.push_back(EffectIn{a.data(), true, {}});
        if (slopes) eff.push_back(EffectIn{b.data(), true, {z.data()}});
        else eff.push_back(EffectIn{b.data(), true, {}});
        if (trial % 3 != 2) eff.push_back(EffectIn{c.data(), true, {}});
        HostDesign d = make_design(n, eff);
        const double* wp = slopes ? w.data() : nullptr;
        if (slopes) build_reparam(d, wp);   // loadings whitened in place, as the solver does
        PrecondCfg cfg;
        cfg.core_dense_max = (trial % 2) ? 8 : 64;
        cfg.core_min_frac = (trial % 4 < 2) ? 0.0 : 0.3;
        cfg.max_rounds = 64;
        BuildResult br = build_preconditioner(d, wp, cfg);
        if (br.kind != 1) return fail("additive Schwarz expected", trial);
        const SchwarzHost& S = br.schwarz;
        if (trial % 6 == 0 || big) {
            setenv("WITHIN_HOST_THREADS", "1", 1);
            BuildResult one = build_preconditioner(d, wp, cfg);
            unsetenv("WITHIN_HOST_THREADS");
            if (image_hash(one.schwarz) != image_hash(S) || one.n_warnings != br.n_warnings)
                return fail("host image depends on the number of host threads", trial);
        }
        const uint32_t n_loc = (uint32_t)S.glob.size(), n_red = S.n_red;
        // index ranges
        for (uint32_t g : S.glob)
            if (g >= S.n_dofs) return fail("glob", trial);
        for (uint32_t e : S.elim_slot)
            if (e >= n_loc) return fail("elim_slot", trial);
        for (uint32_t k : S.c_col)
            if ((k & 0x7fffffffu) >= n_red) return fail("c_col", trial);
        for (uint32_t e : S.ct_col)
            if (e >= n_loc) return fail("ct_col", trial);
        if (S.c_ptr.back() != S.c_col.size() || S.ct_ptr.back() != S.ct_col.size())
            return fail("C pointers", trial);
        for (uint32_t w : S.fwd_col)
            if (w >= n_red) return fail("fwd_col", trial);
        for (uint32_t w : S.bwd_col)
            if (w >= n_red) return fail("bwd_col", trial);
        std::vector<int> seen(n_loc, 0);
        for (uint32_t j : S.dof_slot) {
            if (j >= n_loc || seen[j]++) return fail("dof_slot is not a permutation of the local slots", trial);
        }
        // round of every reduced slot that has factor rows
        std::vector<int> round_of(n_red, -1);
        for (uint32_t r = 0; r < S.n_rounds; ++r)
            for (uint32_t i = S.fwd_round_ptr[r]; i < S.fwd_round_ptr[r + 1]; ++i) {
                if (round_of[S.fwd_row[i]] != -1) return fail("slot in two rounds", trial);
                round_of[S.fwd_row[i]] = (int)r;
            }
        std::vector<int> bwd_empty(n_red, 1);
        for (uint32_t r = 0; r < S.n_rounds; ++r)
            for (uint32_t i = S.bwd_round_ptr[r]; i < S.bwd_round_ptr[r + 1]; ++i)
                bwd_empty[S.bwd_row[i]] = S.bwd_ptr[i + 1] == S.bwd_ptr[i];
        for (uint32_t r = 0; r < S.n_rounds; ++r) {
            for (uint32_t i = S.fwd_round_ptr[r]; i < S.fwd_round_ptr[r + 1]; ++i) {
                ++rows_checked;
                for (uint32_t q = S.fwd_ptr[i]; q < S.fwd_ptr[i + 1]; ++q) {
                    const int rw = round_of[S.fwd_col[q]];
                    if (rw < 0 || rw >= (int)r) return fail("forward row reads its own or a later round", trial);
                }
            }
            for (uint32_t i = S.bwd_round_ptr[r]; i < S.bwd_round_ptr[r + 1]; ++i) {
                if (S.bwd_row[i] != S.fwd_row[i]) return fail("backward rows out of step", trial);
                for (uint32_t q = S.bwd_ptr[i]; q < S.bwd_ptr[i + 1]; ++q) {
                    const uint32_t u = S.bwd_col[q];
                    if (round_of[u] <= (int)r && !bwd_empty[u])
                        return fail("backward row reads a row updated in its own or an earlier round", trial);
                }
            }
        }
        rounds_seen += S.n_rounds;
        for (int32_t m : S.mode) not_laplacian += m != 0;
    }
    if (not_laplacian == 0) {
        printf("FAIL no grounded or cover subdomain was built\n");
        return 1;
    }
    if (rounds_seen == 0) {
        printf("FAIL no round-scheduled factor was built\n");
        return 1;
    }
    printf("schwarz ok: %llu rounds, %llu forward rows checked, %llu grounded or cover subdomains\n",
           (unsigned long long)rounds_seen, (unsigned long long)rows_checked, (unsigned long long)not_laplacian);
    return 0;
}
