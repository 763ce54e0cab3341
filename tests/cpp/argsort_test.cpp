// The locality sort's stable argsort (host_design.cpp stable_argsort_u32)
// against std::stable_sort on random keys, on both sides of its size cut-off
// and for level counts on both sides of the one-pass / two-pass split.
#include <algorithm>
#include <cstdio>
#include <numeric>
#include <random>
#include <vector>

#include "host.hpp"

using namespace wgpu;

int main() {
    std::mt19937_64 rng(11);
    const size_t sizes[] = {1000, ((size_t)1 << 20) + 123};
    const size_t levels[] = {1, 7, 2048, 2049, 100000, 3000000};
    int cases = 0;
    for (size_t n : sizes)
        for (size_t L : levels) {
            std::vector<uint32_t> key(n);
            // skewed keys: many repeats, some levels absent
            for (auto& k : key) k = (uint32_t)((rng() % L) * (rng() % 4 == 0 ? 0 : 1));
            std::vector<uint32_t> want(n), got(n);
            std::iota(want.begin(), want.end(), 0u);
            std::stable_sort(want.begin(), want.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
            stable_argsort_u32(key.data(), n, L, got.data());
            if (got != want) {
                printf("FAIL n %zu levels %zu\n", n, L);
                return 1;
            }
            ++cases;
        }
    printf("argsort ok %d\n", cases);
    return 0;
}
