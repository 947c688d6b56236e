// host_pool.h -- a small persistent pool of host threads for the layout
// conversion between the reference's half-box grids and the packed sphere.
//
// The reference's orbitals live on the full half-box FFT grid, of which the
// plane-wave sphere is a few percent; the rest is zeros.  Gathering the
// sphere on the host and moving only it over PCIe (pinned), then writing the
// zeros on the host, replaces pageable copies of every grid point.  Those
// host loops are memory-bound, so they run on several threads.
//
// One job runs at a time (start() takes the pool, wait() releases it); the
// calling thread works on the job too inside wait().  Thread count: the
// CPUs this process may run on, at most 16, or CPSD_B200_HOST_THREADS.
#pragma once

#include <sched.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdlib>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace cpsd_host {

class Pool {
public:
    // The process-wide pool (created on first use; a forked child makes its own).
    static Pool &get()
    {
        static std::mutex mu;
        static Pool *pool = nullptr;
        std::lock_guard<std::mutex> lk(mu);
        if (!pool || pool->pid_ != getpid()) pool = new Pool();  // the threads live until exit
        return *pool;
    }

    int threads() const { return (int)workers_.size() + 1; }

    // Start fn(i), i < n, on the worker threads; the caller must call wait().
    void start(int n, std::function<void(int)> fn)
    {
        job_mu_.lock();
        std::lock_guard<std::mutex> lk(mu_);
        fn_ = std::move(fn);
        n_ = n;
        done_ = 0;
        ++gen_;
        ctr_.store((unsigned long long)(gen_ & 0xffffffffu) << 32);
        cv_.notify_all();
    }

    // Work on the started job from this thread, then wait for the rest.
    void wait()
    {
        unsigned gen;
        int n;
        {
            std::lock_guard<std::mutex> lk(mu_);
            gen = (unsigned)gen_;
            n = n_;
        }
        const int did = drain(gen, n);
        std::unique_lock<std::mutex> lk(mu_);
        done_ += did;
        done_cv_.wait(lk, [&] { return done_ >= n_; });
        fn_ = nullptr;
        lk.unlock();
        job_mu_.unlock();
    }

    void run(int n, std::function<void(int)> fn)
    {
        start(n, std::move(fn));
        wait();
    }

private:
    Pool() : pid_(getpid())
    {
        int nt = 16;
        cpu_set_t set;
        if (sched_getaffinity(0, sizeof(set), &set) == 0) nt = std::min(nt, CPU_COUNT(&set));
        if (const char *e = std::getenv("CPSD_B200_HOST_THREADS")) nt = std::atoi(e);
        nt = std::max(1, std::min(nt, 256));
        for (int t = 1; t < nt; ++t) workers_.emplace_back([this] { loop(); });
        for (auto &w : workers_) w.detach();
    }

    // Claim items of job `gen` (n items) until none is left.  The counter
    // carries the job number, and a claim only succeeds while it still
    // names job `gen`, so a late thread neither runs nor uses up an item of
    // a later job.
    int drain(unsigned gen, int n)
    {
        int did = 0;
        unsigned long long c = ctr_.load();
        for (;;) {
            if ((unsigned)(c >> 32) != gen || (long long)(c & 0xffffffffu) >= n) break;
            if (!ctr_.compare_exchange_weak(c, c + 1)) continue;  // c reloaded
            fn_((int)(c & 0xffffffffu));
            ++did;
            c = ctr_.load();
        }
        return did;
    }

    void loop()
    {
        unsigned long seen = 0;
        for (;;) {
            int n;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                n = n_;
            }
            const int did = drain((unsigned)(seen & 0xffffffffu), n);
            if (did) {
                std::lock_guard<std::mutex> lk(mu_);
                done_ += did;
                if (done_ >= n_) done_cv_.notify_all();
            }
        }
    }

    const pid_t pid_;
    std::vector<std::thread> workers_;
    std::mutex job_mu_;  // one job at a time
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::function<void(int)> fn_;
    std::atomic<unsigned long long> ctr_{0};  // job number << 32 | next item
    int n_ = 0, done_ = 0;
    unsigned long gen_ = 0;
};

}  // namespace cpsd_host
