// The host pool of the set-up (host_pool.hpp): every item runs once, jobs
// posted from inside items and from several caller threads complete, the
// lowest failing index's exception is the one rethrown, and
// WITHIN_HOST_THREADS=1 runs the items in order on the caller.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "host_pool.hpp"

using namespace wgpu;

static int fail(const char* what) {
    printf("FAIL %s\n", what);
    return 1;
}

int main() {
    // every item once
    {
        std::vector<std::atomic<int>> hit(10000);
        for (auto& h : hit) h = 0;
        par_for_each(hit.size(), [&](size_t i) { hit[i].fetch_add(1); });
        for (auto& h : hit)
            if (h.load() != 1) return fail("each item once");
    }
    // nested jobs: outer items post inner jobs
    {
        std::vector<long> out(64, 0);
        par_for_each(out.size(), [&](size_t i) {
            std::vector<long> part(100, 0);
            par_for_each(part.size(), [&](size_t j) { part[j] = (long)(i * 1000 + j); });
            long s = 0;
            for (long v : part) s += v;
            out[i] = s;
        });
        for (size_t i = 0; i < out.size(); ++i)
            if (out[i] != (long)(i * 1000 * 100 + 99 * 100 / 2)) return fail("nested jobs");
    }
    // several callers side by side (builds of many designs on their own threads)
    {
        std::vector<std::thread> th;
        std::atomic<int> bad{0};
        for (int t = 0; t < 6; ++t)
            th.emplace_back([&, t] {
                for (int rep = 0; rep < 50; ++rep) {
                    std::vector<int> v(257, 0);
                    par_for_each(v.size(), [&](size_t i) { v[i] = (int)i + t; });
                    for (size_t i = 0; i < v.size(); ++i)
                        if (v[i] != (int)i + t) bad.fetch_add(1);
                }
            });
        for (auto& x : th) x.join();
        if (bad.load()) return fail("concurrent callers");
    }
    // the lowest failing index is rethrown, after every item ran
    {
        std::atomic<int> ran{0};
        std::string msg;
        try {
            par_for_each(200, [&](size_t i) {
                ran.fetch_add(1);
                if (i == 17 || i == 150 || i == 5) throw std::runtime_error("item " + std::to_string(i));
            });
        } catch (const std::runtime_error& e) {
            msg = e.what();
        }
        if (msg != "item 5") return fail("lowest failing index");
        if (ran.load() != 200) return fail("every item ran");
    }
    // WITHIN_HOST_THREADS=1: in order on the caller
    {
        setenv("WITHIN_HOST_THREADS", "1", 1);
        const std::thread::id me = std::this_thread::get_id();
        std::vector<size_t> order;
        bool same = true;
        par_for_each(100, [&](size_t i) {
            order.push_back(i);
            same = same && std::this_thread::get_id() == me;
        });
        unsetenv("WITHIN_HOST_THREADS");
        if (!same) return fail("serial on the caller");
        for (size_t i = 0; i < order.size(); ++i)
            if (order[i] != i) return fail("serial order");
    }
    printf("pool ok\n");
    return 0;
}
