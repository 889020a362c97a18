// host_pool.h -- a small persistent pool of host threads for the row-wise file
// I/O of the drop-in entry (DEM reads, .geo merges), so that a call does not
// pay for starting and joining threads.  Internal to libsrg_bp.so.
#pragma once
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace srg {
namespace detail {

class HostPool {
   public:
    // fn(i) for i in [0, n) on the pool's threads and the caller's; returns when
    // every task has run.  Safe to call from several host threads at once.
    void run(int n, const std::function<void(int)> &fn) {
        if (n <= 0) return;
        auto job = std::make_shared<Job>();
        job->fn = &fn;
        job->n = n;
        {
            std::lock_guard<std::mutex> g(mu_);
            for (int i = 0; i < std::min(n - 1, (int)th_.size()); ++i) q_.push_back(job);
        }
        cv_.notify_all();
        work(*job);  // the caller takes tasks too
        std::unique_lock<std::mutex> lk(job->mu);
        job->cv.wait(lk, [&] { return job->done.load() == job->n; });
    }

    // The process-wide pool (made anew in a forked child, whose threads are gone).
    static HostPool &get() {
        static std::mutex m;
        static HostPool *pool = nullptr;
        static pid_t owner = 0;
        std::lock_guard<std::mutex> g(m);
        if (!pool || owner != getpid()) {
            pool = new HostPool();  // a forked child's stale pool is left behind
            owner = getpid();
        }
        return *pool;
    }

    static int threads() {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        return (int)std::min(hw, 16u);
    }

   private:
    struct Job {
        const std::function<void(int)> *fn = nullptr;
        int n = 0;
        std::atomic<int> next{0}, done{0};
        std::mutex mu;
        std::condition_variable cv;
    };

    HostPool() {
        const int nt = threads() - 1;
        for (int i = 0; i < nt; ++i) {
            try {
                th_.emplace_back([this] { loop(); });
            } catch (...) {
                break;  // fewer workers; the caller still runs every task
            }
        }
        for (auto &t : th_) t.detach();
    }

    // Tasks are claimed by index; a queue entry popped after the job finished
    // claims nothing and never touches fn.
    static void work(Job &j) {
        for (int i = j.next.fetch_add(1); i < j.n; i = j.next.fetch_add(1)) {
            (*j.fn)(i);
            if (j.done.fetch_add(1) + 1 == j.n) {
                std::lock_guard<std::mutex> g(j.mu);
                j.cv.notify_all();
            }
        }
    }

    void loop() {
        for (;;) {
            std::shared_ptr<Job> j;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return !q_.empty(); });
                j = q_.front();
                q_.pop_front();
            }
            work(*j);
        }
    }

    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::shared_ptr<Job>> q_;
    std::vector<std::thread> th_;
};

}  // namespace detail
}  // namespace srg
