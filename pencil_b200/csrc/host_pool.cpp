// host_pool.cpp - the host worker threads of the scene upload (validation,
// conversion, 4-wide collapse). Threads are started once per process and
// sleep between jobs: an upload runs several short parallel loops, and
// starting threads for each of them cost more than the loops themselves.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include <unistd.h>

#include "host_internal.h"

namespace pgpu {

namespace {

class HostPool {
public:
    explicit HostPool(int workers) {
        for (int k = 0; k < workers; ++k) std::thread([this] { loop(); }).detach();
        n_workers_ = workers;
    }

    int threads() const { return n_workers_ + 1; }

    // Runs task(0 .. n-1) on the workers and the calling thread; returns when
    // all have finished. One job at a time (callers queue on job_mu_).
    void run(int n, const std::function<void(int)>& task) {
        std::lock_guard<std::mutex> job(job_mu_);
        {
            std::lock_guard<std::mutex> lk(mu_);
            task_ = &task;
            n_ = n;
            next_.store(0);
            busy_ = n_workers_;
            ++generation_;
        }
        cv_.notify_all();
        drain();
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [this] { return busy_ == 0; });
        task_ = nullptr;
    }

private:
    void drain() {
        for (int t; (t = next_.fetch_add(1)) < n_;) (*task_)(t);
    }
    void loop() {
        unsigned long long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return generation_ != seen; });
                seen = generation_;
            }
            drain();
            std::lock_guard<std::mutex> lk(mu_);
            if (--busy_ == 0) done_cv_.notify_one();
        }
    }

    int n_workers_ = 0;
    std::mutex job_mu_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)>* task_ = nullptr;
    std::atomic<int> next_{0};
    int n_ = 0;
    int busy_ = 0;
    unsigned long long generation_ = 0;
};

HostPool& pool() {
    // Never destroyed: its threads sleep until the process ends. A child made
    // by fork() has none of its parent's threads, so it starts its own pool
    // (the parent's object is left as it is).
    static std::mutex mu;
    static HostPool* p = nullptr;
    static pid_t owner = 0;
    std::lock_guard<std::mutex> lk(mu);
    if (!p || owner != getpid()) {
        p = new HostPool(
            std::max(0, std::min(16, (int)std::max(1u, std::thread::hardware_concurrency())) - 1));
        owner = getpid();
    }
    return *p;
}

}  // namespace

int host_threads() { return pool().threads(); }

void host_run(int n, const std::function<void(int)>& task) {
    if (n <= 0) return;
    if (n == 1 || host_threads() == 1) {
        for (int t = 0; t < n; ++t) task(t);
        return;
    }
    pool().run(n, task);
}

}  // namespace pgpu
