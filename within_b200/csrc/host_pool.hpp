// host_pool.hpp -- the host thread pool of the set-up (preconditioner build,
// design lowering): par_for_each over indexed items.
#pragma once
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdlib>
#include <exception>
#include <mutex>
#include <thread>
#include <type_traits>
#include <vector>

namespace wgpu {

// A process-wide pool of host worker threads, created on first use and kept
// for the life of the process (up to 15 workers: 16 threads with the
// caller; WITHIN_HOST_THREADS, read at every job, lowers the total).  A job is n indexed items;
// the caller posts it, works on its items itself and waits only for items
// already running on workers, so jobs posted from inside other jobs' items
// (a build per design, a domain per thread) cannot deadlock.
class HostPool {
  public:
    struct Job {
        void (*call)(void*, size_t);
        void* ctx;
        size_t n;
        std::atomic<size_t> next{0};
        std::atomic<size_t> done{0};
        size_t users = 0;       // workers holding the job (guarded by the pool mutex)
        size_t max_users = 0;   // at most this many workers join the caller
        std::vector<std::exception_ptr>* err;
    };
    static HostPool& get() {
        static HostPool* p = new HostPool();   // never destroyed: workers outlive static destructors
        return *p;
    }
    size_t threads() const { return n_threads_; }
    void run(Job& j) {
        {
            std::lock_guard<std::mutex> g(mu_);
            jobs_.push_back(&j);
        }
        cv_.notify_all();
        work_on(j);
        {
            std::lock_guard<std::mutex> g(mu_);
            jobs_.erase(std::find(jobs_.begin(), jobs_.end(), &j));
        }
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return j.done.load() == j.n && j.users == 0; });
    }

  private:
    HostPool() {
        const size_t cap = std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
        n_threads_ = cap;
        for (size_t t = 1; t < cap; ++t) std::thread([this] { worker(); }).detach();
    }
    static void work_on(Job& j) {
        for (size_t i; (i = j.next.fetch_add(1)) < j.n;) {
            try {
                j.call(j.ctx, i);
            } catch (...) {
                (*j.err)[i] = std::current_exception();
            }
            j.done.fetch_add(1);
        }
    }
    void worker() {
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            Job* j = nullptr;
            cv_.wait(lk, [&] {
                for (Job* x : jobs_)
                    if (x->next.load() < x->n && x->users < x->max_users) {
                        j = x;
                        return true;
                    }
                return false;
            });
            ++j->users;
            lk.unlock();
            work_on(*j);
            lk.lock();
            --j->users;
            if (j->done.load() == j->n && j->users == 0) done_cv_.notify_all();
        }
    }
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::vector<Job*> jobs_;
    size_t n_threads_ = 1;
};

// f(i) for i in [0, n) on the host pool.  Every f(i) writes only its own
// outputs, so the result does not depend on the schedule; the exception of
// the lowest failing index is rethrown, as the sequential loop would have
// thrown it.
template <class F>
inline void par_for_each(size_t n, F&& f) {
    size_t cap = 16;
    if (const char* e = std::getenv("WITHIN_HOST_THREADS")) cap = (size_t)std::max(1, std::atoi(e));
    if (n <= 1 || cap <= 1) {
        for (size_t i = 0; i < n; ++i) f(i);
        return;
    }
    HostPool& pool = HostPool::get();
    if (pool.threads() <= 1) {
        for (size_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::vector<std::exception_ptr> err(n);
    using Fn = std::remove_reference_t<F>;
    HostPool::Job j;
    j.call = [](void* c, size_t i) { (*static_cast<Fn*>(c))(i); };
    j.ctx = (void*)&f;
    j.n = n;
    j.max_users = std::min(cap, pool.threads()) - 1;
    j.err = &err;
    pool.run(j);
    for (auto& e : err)
        if (e) std::rethrow_exception(e);
}

}  // namespace wgpu
