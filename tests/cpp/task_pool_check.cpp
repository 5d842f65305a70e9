// Test driver: the host task pool (hpgl_b200/csrc/task_pool.cpp).  Each
// check returns the number of failures; tpc_all runs them all.
#include <atomic>
#include <stdexcept>
#include <thread>
#include <vector>

#include "../../hpgl_b200/csrc/task_pool.h"

using namespace hpgl_b200;

// pool_for covers [0, n) exactly once for any thread count and grain.
extern "C" int tpc_cover(void) {
    int bad = 0;
    for (int threads : {1, 2, 3, 8, 33})
        for (long long n : {0LL, 1LL, 7LL, 4096LL, 100003LL}) {
            std::vector<std::atomic<int>> hit((size_t)n);
            for (auto &h : hit) h = 0;
            pool_for(n, threads, [&](long long lo, long long hi) {
                for (long long i = lo; i < hi; ++i) hit[(size_t)i]++;
            }, 100);
            for (auto &h : hit) bad += h.load() != 1;
        }
    return bad;
}

// A task that itself runs a pool_for and waits (nested groups) completes.
extern "C" int tpc_nested(void) {
    std::atomic<long long> sum{0};
    pool_for(64, 8, [&](long long lo, long long hi) {
        for (long long i = lo; i < hi; ++i)
            pool_for(1000, 4, [&](long long a, long long b) { sum += b - a; }, 10);
    }, 1);
    return sum.load() == 64 * 1000 ? 0 : 1;
}

// An exception thrown by any chunk reaches the caller once every chunk has
// finished, and the pool keeps working afterwards.
extern "C" int tpc_exception(void) {
    int bad = 0;
    for (int which : {0, 5}) {
        std::atomic<int> done{0};
        bool caught = false;
        try {
            pool_for(8, 8, [&](long long lo, long long) {
                if (lo == which) throw std::runtime_error("chunk failed");
                done++;
            }, 1);
        } catch (const std::runtime_error &) {
            caught = true;
        }
        bad += !caught;
        bad += done.load() != 7;
    }
    std::atomic<int> after{0};
    pool_for(100, 8, [&](long long lo, long long hi) { after += (int)(hi - lo); }, 1);
    bad += after.load() != 100;
    return bad;
}

// Several threads run pool_for at once, each on its own data.
extern "C" int tpc_concurrent(void) {
    std::atomic<int> bad{0};
    std::vector<std::thread> callers;
    for (int c = 0; c < 6; ++c)
        callers.emplace_back([&, c] {
            for (int rep = 0; rep < 20; ++rep) {
                std::atomic<long long> sum{0};
                const long long n = 1000 + 37 * c + rep;
                pool_for(n, 5, [&](long long lo, long long hi) {
                    long long s = 0;
                    for (long long i = lo; i < hi; ++i) s += i;
                    sum += s;
                }, 16);
                if (sum.load() != n * (n - 1) / 2) bad++;
            }
        });
    for (auto &t : callers) t.join();
    return bad.load();
}

// Sub-tasks submitted by running tasks of the same group are waited for.
extern "C" int tpc_subtasks(void) {
    TaskGroup g;
    std::atomic<int> leaves{0};
    std::function<void(int)> spawn = [&](int depth) {
        if (depth == 0) {
            leaves++;
            return;
        }
        task_submit(g, [&, depth] { spawn(depth - 1); });
        task_submit(g, [&, depth] { spawn(depth - 1); });
    };
    task_pool_reserve(4);
    spawn(10);
    task_wait(g);
    return leaves.load() == 1024 ? 0 : 1;
}

extern "C" int tpc_all(void) { return tpc_cover() + tpc_nested() + tpc_exception() + tpc_concurrent() + tpc_subtasks(); }
