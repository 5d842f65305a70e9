// Persistent host worker threads (task_pool.h).
#include "task_pool.h"

#include <condition_variable>
#include <deque>
#include <thread>
#include <utility>
#include <vector>

namespace hpgl_b200 {

namespace {

struct Task {
    TaskGroup *group;
    std::function<void()> fn;
};

// One process-wide pool.  It is never destroyed: worker threads blocked on
// its condition variable at exit must not outlive it.
struct Pool {
    std::mutex mu;
    std::condition_variable has_task;   // workers wait here
    std::condition_variable group_done; // waiting callers wait here
    std::deque<Task> queue;
    int workers = 0;

    void run(Task &t) {
        try {
            t.fn();
        } catch (...) {
            std::lock_guard<std::mutex> l(t.group->err_mu);
            if (!t.group->err) t.group->err = std::current_exception();
        }
        t.fn = nullptr;  // release the closure before the group can end
        if (t.group->pending.fetch_sub(1) == 1) {
            std::lock_guard<std::mutex> l(mu);
            group_done.notify_all();
        }
    }

    void worker_loop() {
        std::unique_lock<std::mutex> lk(mu);
        while (true) {
            has_task.wait(lk, [this] { return !queue.empty(); });
            Task t = std::move(queue.front());
            queue.pop_front();
            lk.unlock();
            run(t);
            lk.lock();
        }
    }
};

Pool &pool() {
    static Pool *p = new Pool();
    return *p;
}

}  // namespace

void task_pool_reserve(int n) {
    Pool &p = pool();
    std::lock_guard<std::mutex> l(p.mu);
    const unsigned hc = std::thread::hardware_concurrency();
    const int cap = hc ? 2 * (int)hc : 64;  // never more than twice the host's threads
    if (n > cap) n = cap;
    while (p.workers < n) {
        std::thread([&p] { p.worker_loop(); }).detach();
        ++p.workers;
    }
}

void task_submit(TaskGroup &g, std::function<void()> f) {
    Pool &p = pool();
    g.pending.fetch_add(1);
    {
        std::lock_guard<std::mutex> l(p.mu);
        p.queue.push_back(Task{&g, std::move(f)});
    }
    p.has_task.notify_one();
    p.group_done.notify_all();  // waiting callers run queued tasks too
}

void task_wait(TaskGroup &g) {
    Pool &p = pool();
    std::unique_lock<std::mutex> lk(p.mu);
    while (g.pending.load() > 0) {
        if (!p.queue.empty()) {
            Task t = std::move(p.queue.front());
            p.queue.pop_front();
            lk.unlock();
            p.run(t);
            lk.lock();
        } else {
            p.group_done.wait(lk, [&] { return g.pending.load() == 0 || !p.queue.empty(); });
        }
    }
    lk.unlock();
    std::lock_guard<std::mutex> l(g.err_mu);
    if (g.err) std::rethrow_exception(g.err);
}

}  // namespace hpgl_b200
