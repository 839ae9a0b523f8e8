// Minimal stand-in for oneTBB's parallel_for, used only to compile the reference CPU stereo
// (libs/depth/src/stereo.cpp) for the oracle and the CPU baseline; oneTBB is not installed here.
// A persistent pool of std::threads takes chunks of the range from an atomic counter (dynamic
// scheduling, like TBB's auto partitioner). Thread count: ORACLE_THREADS, else hardware_concurrency.
// Nested calls from a worker run serially. Test infrastructure, not product code.
#pragma once

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdlib>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "tbb/blocked_range.h"

namespace tbb {
namespace stub_detail {

class Pool {
public:
    static Pool& instance() {
        static Pool pool;
        return pool;
    }

    int threads() const { return static_cast<int>(workers_.size()) + 1; }

    // Runs body(c) for every chunk c in [0, chunks), on the pool plus the calling thread.
    void run(std::size_t chunks, const std::function<void(std::size_t)>& body) {
        if (chunks == 0) return;
        if (in_worker() || workers_.empty() || chunks == 1) {
            for (std::size_t c = 0; c < chunks; ++c) body(c);
            return;
        }
        std::lock_guard<std::mutex> serial(run_mutex_);  // one job at a time
        {
            std::lock_guard<std::mutex> lk(m_);
            body_ = &body;
            chunks_ = chunks;
            next_.store(0);
            done_.store(0);
            ++generation_;
        }
        cv_.notify_all();
        in_worker() = true;
        work();
        in_worker() = false;
        std::unique_lock<std::mutex> lk(m_);
        done_cv_.wait(lk, [&] { return done_.load() == chunks_; });
        body_ = nullptr;
    }

private:
    Pool() {
        int n = static_cast<int>(std::thread::hardware_concurrency());
        if (const char* e = std::getenv("ORACLE_THREADS")) n = std::atoi(e);
        n = std::max(1, n);
        for (int i = 1; i < n; ++i) workers_.emplace_back([this] { loop(); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
            ++generation_;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }

    static bool& in_worker() {
        thread_local bool flag = false;
        return flag;
    }

    void work() {
        for (;;) {
            const std::size_t c = next_.fetch_add(1);
            if (c >= chunks_) break;
            (*body_)(c);
            if (done_.fetch_add(1) + 1 == chunks_) {
                std::lock_guard<std::mutex> lk(m_);
                done_cv_.notify_all();
            }
        }
    }

    void loop() {
        in_worker() = true;
        std::size_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || generation_ != seen; });
                if (stop_) return;
                seen = generation_;
                if (body_ == nullptr) continue;
            }
            work();
        }
    }

    std::vector<std::thread> workers_;
    std::mutex run_mutex_, m_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(std::size_t)>* body_ = nullptr;
    std::size_t chunks_ = 0;
    std::atomic<std::size_t> next_{0}, done_{0};
    std::size_t generation_ = 0;
    bool stop_ = false;
};

}  // namespace stub_detail

template <typename T, typename F>
void parallel_for(const blocked_range<T>& range, const F& f) {
    if (range.empty()) return;
    auto& pool = stub_detail::Pool::instance();
    const std::size_t n = range.size();
    const std::size_t chunks = std::min<std::size_t>(n, static_cast<std::size_t>(pool.threads()) * 8);
    const T b = range.begin();
    pool.run(chunks, [&](std::size_t c) {
        const T lo = static_cast<T>(b + static_cast<T>(n * c / chunks));
        const T hi = static_cast<T>(b + static_cast<T>(n * (c + 1) / chunks));
        if (lo < hi) f(blocked_range<T>(lo, hi));
    });
}

template <typename I, typename F>
void parallel_for(I first, I last, const F& f) {
    parallel_for(blocked_range<I>(first, last), [&](const blocked_range<I>& r) {
        for (I i = r.begin(); i != r.end(); ++i) f(i);
    });
}

}  // namespace tbb
