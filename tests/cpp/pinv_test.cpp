// Prints the dense generalised inverse the preconditioner's dense route
// builds (wgpu::dense_pseudo_inverse) for seeded PSD matrices: a connected
// graph Laplacian, a Laplacian of two components, and a strictly diagonally
// dominant SDD matrix.  tests/test_cpu_host.py compares each with numpy's pinv.
#include <cstdio>
#include <random>
#include <vector>

#include "host.hpp"

int main() {
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U(0.1, 2.0);
    const unsigned sizes[] = {5, 37, 200};
    for (unsigned n : sizes)
        for (int kind = 0; kind < 3; ++kind) {
            std::vector<double> a((size_t)n * n, 0.0);
            auto edge = [&](unsigned i, unsigned j, double w) {
                a[(size_t)i * n + j] -= w;
                a[(size_t)j * n + i] -= w;
                a[(size_t)i * n + i] += w;
                a[(size_t)j * n + j] += w;
            };
            const unsigned half = n / 2;
            for (unsigned i = 0; i + 1 < n; ++i) {
                if (kind == 1 && i + 1 == half) continue;   // two components
                edge(i, i + 1, U(rng));
            }
            for (unsigned t = 0; t < 2 * n; ++t) {
                unsigned i = rng() % n, j = rng() % n;
                if (i == j || (kind == 1 && ((i < half) != (j < half)))) continue;
                edge(i, j, U(rng));
            }
            if (kind == 2)
                for (unsigned i = 0; i < n; ++i) a[(size_t)i * n + i] += 0.05 * U(rng);
            const std::vector<double> g = wgpu::dense_pseudo_inverse(n, a);
            printf("case %u %d %zu\n", n, kind, g.size());
            for (double v : a) printf("%.17g ", v);
            printf("\n");
            for (double v : g) printf("%.17g ", v);
            printf("\n");
        }
    printf("pinv done\n");
    return 0;
}
