// Persistent host worker threads for the library's parallel host work
// (planning: covariance boxes, template keys and sort, buckets; staging
// copies).  Work is submitted as tasks of a TaskGroup; whoever waits for a
// group runs queued tasks itself until the group is done, so nested groups
// (a task that submits and waits) and concurrent callers (the bucket thread
// beside the template sort, several serving planners) always make progress,
// and a process without workers (e.g. a forked child) still completes every
// group on the waiting thread.
#pragma once

#include <atomic>
#include <exception>
#include <functional>
#include <mutex>

namespace hpgl_b200 {

struct TaskGroup {
    std::atomic<long long> pending{0};
    std::mutex err_mu;
    std::exception_ptr err;  // first exception a task of the group threw
};

// Makes sure at least `n` worker threads exist (they are never stopped).
void task_pool_reserve(int n);
// Queues f as a task of g.
void task_submit(TaskGroup &g, std::function<void()> f);
// Runs queued tasks until every task of g has finished; rethrows the first
// exception of g's tasks.
void task_wait(TaskGroup &g);

// f(lo, hi) over [0, n) in up to `threads` chunks of at least `grain` items:
// the first chunk on the calling thread, the others as tasks.
template <typename F>
void pool_for(long long n, int threads, F f, long long grain = 4096) {
    if (n <= 0) return;
    long long parts = n / (grain > 0 ? grain : 1) + 1;
    if (parts > threads) parts = threads;
    if (parts < 1) parts = 1;
    if (parts == 1) {
        f(0LL, n);
        return;
    }
    task_pool_reserve((int)parts - 1);
    const long long chunk = (n + parts - 1) / parts;
    TaskGroup g;
    for (long long t = 1; t < parts; ++t) {
        const long long lo = t * chunk, hi = lo + chunk < n ? lo + chunk : n;
        if (lo >= hi) break;
        task_submit(g, [lo, hi, &f] { f(lo, hi); });
    }
    std::exception_ptr own;
    try {
        f(0LL, chunk < n ? chunk : n);
    } catch (...) {
        own = std::current_exception();
    }
    task_wait(g);  // the other chunks reference f: wait for them before leaving
    if (own) std::rethrow_exception(own);
}

}  // namespace hpgl_b200
