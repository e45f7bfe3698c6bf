// copy_pool.h -- a few host threads that split the copy of a force call's
// results from pinned staging into the caller's arrays.
//
// The caller's arrays are ordinary (pageable) memory, so a call's results
// cross the host twice: the DMA into pinned staging, then a CPU copy into
// the caller's arrays.  One core copies at about 10 GB/s, so for a large
// irregular call (65,536 bodies, 3.7 MB of acc, jrk and nnbid) that second
// copy takes longer than the force kernel.  The pool runs it on `parts()`
// threads (the calling thread is part 0).  Idle helpers spin for up to 2 ms
// after each job or arm() (force calls come in quick succession: a
// 1,024-body regular call takes ~1.4 ms), then sleep on a condition
// variable.
//
// NB6_COPY_THREADS sets the number of parts (1 = the calling thread alone);
// the default is min(4, hardware threads / 2).  One pool serves the whole
// library (nb6_copy_pool); its threads start with the first large call and
// stop when the last of the regular and irregular libraries is closed.
#pragma once

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include <unistd.h>

#if defined(__x86_64__) || defined(_M_X64)
#include <immintrin.h>
#define NB6_CPU_PAUSE() _mm_pause()
#else
#define NB6_CPU_PAUSE() std::this_thread::yield()
#endif

class CopyPool {
  public:
    ~CopyPool() { stop(); }

    static int default_parts() {
        if (const char *e = getenv("NB6_COPY_THREADS")) {
            const int n = atoi(e);
            return n < 1 ? 1 : (n > 64 ? 64 : n);
        }
        const int hw = (int)std::thread::hardware_concurrency();
        const int n = hw / 2;
        return n < 1 ? 1 : (n > 4 ? 4 : n);
    }

    // Start nparts - 1 helpers (no-op when already running).
    void start(int nparts) {
        if (!th_.empty() || nparts <= 1) return;
        pid_ = getpid();
        quit_.store(false);
        const unsigned g0 = gen_.load();   // helpers wait for the next generation
        for (int p = 1; p < nparts; ++p) th_.emplace_back(&CopyPool::loop, this, p, g0);
    }

    void stop() {
        if (th_.empty() || getpid() != pid_) return;
        {
            std::lock_guard<std::mutex> lk(mu_);
            quit_.store(true);
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
        th_.clear();
    }

    int parts() const { return (int)th_.size() + 1; }

    // f(p) for p in [0, parts()); p = 0 on the calling thread.  Returns when
    // every part has returned.  Not reentrant: one caller at a time.
    void run(std::function<void(int)> f) {
        if (th_.empty()) {
            f(0);
            return;
        }
        if (getpid() != pid_) {   // a forked child has none of the helpers
            for (int p = 0; p < parts(); ++p) f(p);
            return;
        }
        job_ = std::move(f);
        left_.store((int)th_.size(), std::memory_order_relaxed);
        {
            std::lock_guard<std::mutex> lk(mu_);   // no wake-up lost to a helper going to sleep
            gen_.fetch_add(1, std::memory_order_release);
        }
        cv_.notify_all();
        job_(0);
        while (left_.load(std::memory_order_acquire) > 0) NB6_CPU_PAUSE();
    }

    // Wake sleeping helpers so that they spin, ready for a job, while the
    // caller still waits for the GPU (a futex wake-up can take longer than
    // the copy itself).
    void arm() {
        if (th_.empty() || getpid() != pid_) return;
        {
            std::lock_guard<std::mutex> lk(mu_);
            ++wake_;
        }
        cv_.notify_all();
    }

  private:
    static constexpr long long SPIN_NS = 2000000;   // spin up to 2 ms before sleeping

    void loop(int p, unsigned seen) {
        unsigned woken = 0;
        for (;;) {
            unsigned g = gen_.load(std::memory_order_acquire);
            if (g == seen) {
                const auto t0 = std::chrono::steady_clock::now();
                for (int s = 1; g == seen && !quit_.load(std::memory_order_relaxed); ++s) {
                    NB6_CPU_PAUSE();
                    g = gen_.load(std::memory_order_acquire);
                    if ((s & 63) == 0 &&
                        std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0)
                                .count() > SPIN_NS)
                        break;
                }
            }
            if (quit_.load()) return;
            if (g == seen) {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] {
                    return quit_.load() || gen_.load(std::memory_order_acquire) != seen || wake_ != woken;
                });
                woken = wake_;
                if (quit_.load()) return;
                continue;   // a job or an arm(): spin again
            }
            seen = g;
            job_(p);
            left_.fetch_sub(1, std::memory_order_acq_rel);
        }
    }

    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::atomic<unsigned> gen_{0};
    std::atomic<int> left_{0};
    std::atomic<bool> quit_{false};
    unsigned wake_ = 0;   // under mu_
    pid_t pid_ = 0;       // the process that started the helpers
    std::function<void(int)> job_;
};
