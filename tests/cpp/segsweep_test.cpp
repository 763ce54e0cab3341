// Property test of the warp-range segmented sweep (segsweep.cuh) and its
// planner (SSHostPlan::add): random multi-problem segment layouts with runs
// of empty segments, all-empty problems and segments far longer than a range
// are planned, and the kernel's warp algorithm is executed here lane by lane
// (shuffles, ballots and lane masks emulated on arrays of 32 lanes, ranges in
// a shuffled order so the split finisher varies).  Checks: every segment is
// emitted exactly once with the exact sum of its positions (integer-valued
// doubles), every position is read once, and every bitmap, id-list, empty-list
// and partial-buffer index stays inside its array.
#include "host.hpp"
#include <algorithm>
#include <cstdio>
#include <random>
using namespace wgpu;

static int fail(const char* m, int trial) {
    printf("FAIL %s trial %d\n", m, trial);
    return 1;
}

struct Prob {
    const uint32_t* ptr;
    uint32_t n_seg, pos_base;   // pos_base: offset of the problem's values in vals
};

int main() {
    std::mt19937_64 rng(7);
    for (int trial = 0; trial < 600; ++trial) {
        const int R = trial % 3 == 0 ? 4 : trial % 3 == 1 ? 2 : 1;
        const uint32_t CH = 32u * R;
        const int n_prob = 1 + (int)(rng() % 4);
        std::vector<std::vector<uint32_t>> ptrs(n_prob);
        SSHostPlan hp;
        std::vector<Prob> probs(n_prob);
        std::vector<double> vals;
        std::vector<std::vector<double>> expect(n_prob);
        const uint32_t L = SS_ALIGN * (1 + (uint32_t)(rng() % 4));
        for (int q = 0; q < n_prob; ++q) {
            const uint32_t nseg = (uint32_t)(rng() % 1500);
            auto& ptr = ptrs[q];
            ptr.resize(nseg + 1);
            ptr[0] = (uint32_t)(rng() % 1000);
            const int mode = (int)(rng() % 4);   // 0 mixed, 1 all empty, 2 long, 3 short
            for (uint32_t s = 0; s < nseg; ++s) {
                uint32_t len;
                const uint32_t r = (uint32_t)(rng() % 10);
                if (mode == 1) len = 0;
                else if (mode == 2) len = r < 2 ? 0 : (uint32_t)(rng() % (5 * L));
                else if (mode == 3) len = r < 2 ? 0 : 1 + (uint32_t)(rng() % 3);
                else len = r < 4 ? 0 : r < 8 ? (uint32_t)(rng() % 6) : (uint32_t)(rng() % (3 * L));
                ptr[s + 1] = ptr[s] + len;
            }
            probs[q] = Prob{ptr.data(), nseg, (uint32_t)vals.size()};
            expect[q].assign(nseg, 0.0);
            for (uint32_t s = 0; s < nseg; ++s)
                for (uint32_t p = ptr[s]; p < ptr[s + 1]; ++p) {
                    const double v = (double)(int64_t)(rng() % 2001) - 1000.0;
                    expect[q][s] += v;
                    vals.push_back(v);
                }
            hp.add((uint32_t)q, ptr.data(), nseg, L);
        }
        // positions of every problem are contiguous in vals from pos_base
        auto value = [&](uint32_t q, uint32_t P, int trial_) -> double {
            const Prob& pr = probs[q];
            const uint32_t rel = P - pr.ptr[0];
            if (P < pr.ptr[0] || rel >= pr.ptr[pr.n_seg] - pr.ptr[0]) {
                fail("value index", trial_);
                exit(1);
            }
            return vals[pr.pos_base + rel];
        };
        std::vector<std::vector<int>> emitted(n_prob);
        std::vector<std::vector<double>> got(n_prob);
        for (int q = 0; q < n_prob; ++q) {
            emitted[q].assign(probs[q].n_seg, 0);
            got[q].assign(probs[q].n_seg, 0.0);
        }
        std::vector<int> reads(vals.size(), 0);
        const size_t nr = hp.ranges.size();
        std::vector<double> head(nr, 0.0), tail(std::max<size_t>(1, hp.splits.size()), 0.0);
        std::vector<unsigned> counters(std::max<size_t>(1, hp.splits.size()), 0);
        auto emit = [&](uint32_t q, uint32_t seg, double s) {
            if (seg >= probs[q].n_seg) {
                fail("emit id", trial);
                exit(1);
            }
            emitted[q][seg]++;
            got[q][seg] = s;
        };
        std::vector<size_t> order(nr);
        for (size_t i = 0; i < nr; ++i) order[i] = i;
        std::shuffle(order.begin(), order.end(), rng);
        for (size_t oi = 0; oi < nr; ++oi) {
            const uint32_t r = (uint32_t)order[oi];
            const SSRange rg = hp.ranges[r];
            for (uint32_t e = rg.e_lo; e < rg.e_hi; ++e) {
                if (e >= hp.empties.size()) return fail("empty index", trial);
                emit(rg.problem, hp.empties[e], 0.0);
            }
            uint32_t o_base = rg.o0 - (rg.head_split < 0 ? 1u : 0u);
            double carry = 0.0;
            bool cseen = false;
            for (uint32_t c = rg.p0; c < rg.p1; c += CH) {
                const uint32_t cn = c + CH;
                uint32_t fl[32], nxt[32];
                int nval[32];
                double cv[32][4];
                for (int lane = 0; lane < 32; ++lane) {
                    const size_t wi = (size_t)rg.word0 + (c - rg.p0) / 32u + ((uint32_t)lane * R) / 32u;
                    if (wi >= hp.bits.size()) return fail("bitmap index", trial);
                    const uint32_t word = hp.bits[wi];
                    const uint32_t P0 = c + (uint32_t)lane * R;
                    nval[lane] = P0 >= rg.p1 ? 0 : (int)std::min<uint32_t>(R, rg.p1 - P0);
                    fl[lane] = (word >> (((uint32_t)lane * R) & 31u)) & ((1u << R) - 1u);
                    fl[lane] &= (1u << nval[lane]) - 1u;
                    for (int i = 0; i < R; ++i) {
                        const uint32_t P = P0 + i;
                        if (P < rg.p1) {
                            cv[lane][i] = value(rg.problem, P, trial);
                            reads[probs[rg.problem].pos_base + (P - probs[rg.problem].ptr[0])]++;
                        } else {
                            cv[lane][i] = 0.0;
                        }
                    }
                }
                for (int lane = 0; lane < 32; ++lane) {
                    nxt[lane] = lane < 31 ? (fl[lane + 1] & 1u) : 0u;
                    if (lane == 31 && cn < rg.p1) {
                        const size_t wi = (size_t)rg.word0 + (cn - rg.p0) / 32u;
                        if (wi >= hp.bits.size()) return fail("lookahead index", trial);
                        nxt[lane] = hp.bits[wi] & 1u;
                    }
                }
                double tv[32];
                bool tf[32];
                for (int lane = 0; lane < 32; ++lane) {
                    tv[lane] = 0.0;
                    for (int i = 0; i < R; ++i) {
                        if ((fl[lane] >> i) & 1u) tv[lane] = cv[lane][i];
                        else tv[lane] += cv[lane][i];
                    }
                    tf[lane] = fl[lane] != 0u;
                }
                for (int d = 1; d < 32; d <<= 1) {
                    double up[32];
                    bool uf[32];
                    for (int lane = 0; lane < 32; ++lane) {
                        up[lane] = lane >= d ? tv[lane - d] : tv[lane];
                        uf[lane] = lane >= d ? tf[lane - d] : tf[lane];
                    }
                    for (int lane = 0; lane < 32; ++lane)
                        if (lane >= d && !tf[lane]) {
                            tv[lane] += up[lane];
                            tf[lane] = uf[lane];
                        }
                }
                double run[32];
                bool seen[32];
                unsigned ballot[4] = {0, 0, 0, 0};
                for (int i = 0; i < R; ++i)
                    for (int lane = 0; lane < 32; ++lane)
                        if ((fl[lane] >> i) & 1u) ballot[i] |= 1u << lane;
                uint32_t total = 0;
                for (int i = 0; i < R; ++i) total += (uint32_t)__builtin_popcount(ballot[i]);
                for (int lane = 0; lane < 32; ++lane) {
                    bool exf = lane > 0 ? tf[lane - 1] : false;
                    run[lane] = lane > 0 ? tv[lane - 1] : 0.0;
                    if (!exf) run[lane] = carry + run[lane];
                    seen[lane] = exf || cseen;
                    const unsigned lt = (1u << lane) - 1u;
                    uint32_t cnt = 0;
                    for (int i = 0; i < R; ++i) cnt += (uint32_t)__builtin_popcount(ballot[i] & lt);
                    for (int i = 0; i < R; ++i) {
                        if (i >= nval[lane]) continue;
                        if ((fl[lane] >> i) & 1u) {
                            run[lane] = cv[lane][i];
                            seen[lane] = true;
                            ++cnt;
                        } else {
                            run[lane] += cv[lane][i];
                        }
                        const uint32_t P = c + (uint32_t)lane * R + i;
                        const bool at_end = P + 1 == rg.p1;
                        const bool nstart = i + 1 < R ? ((fl[lane] >> (i + 1)) & 1u) != 0 : nxt[lane] != 0;
                        if (at_end || nstart) {
                            if (!seen[lane]) {
                                head[r] = run[lane];
                            } else if (at_end && rg.tail_split >= 0) {
                                if ((size_t)rg.tail_split >= hp.splits.size()) return fail("tail index", trial);
                                tail[rg.tail_split] = run[lane];
                            } else {
                                const uint32_t o = o_base + cnt;
                                uint32_t seg = o;
                                if (rg.nz_off != SS_IDENTITY) {
                                    if ((size_t)rg.nz_off + o >= hp.nz_ids.size()) return fail("nz index", trial);
                                    seg = hp.nz_ids[rg.nz_off + o];
                                }
                                emit(rg.problem, seg, run[lane]);
                            }
                        }
                    }
                }
                carry = run[31];
                cseen = seen[31];
                o_base += total;
            }
            const int ids[2] = {rg.head_split, rg.tail_split};
            for (int j = 0; j < 2; ++j) {
                const int id = ids[j];
                if (id < 0) continue;
                const SSSplit sp = hp.splits[id];
                if (sp.r0 > r || sp.r1 < r) return fail("split range", trial);
                const unsigned prev = counters[id]++;
                if (prev == sp.r1 - sp.r0) {
                    double acc[32];
                    for (int lane = 0; lane < 32; ++lane) {
                        acc[lane] = 0.0;
                        for (uint32_t t = sp.r0 + 1 + lane; t <= sp.r1; t += 32) acc[lane] += head[t];
                    }
                    for (int o = 16; o > 0; o >>= 1) {
                        double nx[32];
                        for (int lane = 0; lane < 32; ++lane) nx[lane] = acc[lane] + acc[lane ^ o];
                        for (int lane = 0; lane < 32; ++lane) acc[lane] = nx[lane];
                    }
                    emit(sp.problem, sp.seg, tail[id] + acc[0]);
                    counters[id] = 0;
                }
            }
        }
        for (int q = 0; q < n_prob; ++q)
            for (uint32_t s = 0; s < probs[q].n_seg; ++s) {
                if (emitted[q][s] != 1) {
                    printf("seg %u of problem %d emitted %d times (len %u)\n", s, q, emitted[q][s],
                           ptrs[q][s + 1] - ptrs[q][s]);
                    return fail("emit count", trial);
                }
                if (got[q][s] != expect[q][s]) return fail("sum", trial);
            }
        for (size_t i = 0; i < reads.size(); ++i)
            if (reads[i] != 1) return fail("read count", trial);
        for (auto c : counters)
            if (c != 0) return fail("counter reset", trial);
        for (const auto& rg : hp.ranges)
            if ((rg.p0 - ptrs[rg.problem][0]) % SS_ALIGN != 0 || rg.p1 - rg.p0 > L) return fail("range shape", trial);
    }
    printf("segsweep ok\n");
}
