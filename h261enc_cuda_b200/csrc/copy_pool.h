/* Host copy workers for the staging arena.
 *
 * A batch of pictures submitted in one call is copied into the pinned
 * staging arena by a small persistent pool: every plane copy is cut into
 * pieces of at most kPiece bytes, the pieces are taken from one atomic
 * counter by the workers and by the calling thread, and the call returns
 * when the last piece is done.  Workers sleep on a condition variable
 * between batches. */
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace h261b {

struct CopyJob {
    uint8_t *dst;
    const uint8_t *src;
    size_t bytes;
};

class CopyPool {
  public:
    static constexpr size_t kPiece = 64 << 10;

    explicit CopyPool(int threads)
    {
        for (int i = 0; i < threads; i++)
            workers_.emplace_back([this] { loop(); });
    }

    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (std::thread &t : workers_)
            t.join();
    }

    CopyPool(const CopyPool &) = delete;
    CopyPool &operator=(const CopyPool &) = delete;

    int threads() const { return (int)workers_.size(); }

    /* copy every job; returns when all bytes are in place */
    void run(const std::vector<CopyJob> &jobs)
    {
        size_t total = 0;
        for (const CopyJob &j : jobs)
            total += j.bytes;
        if (workers_.empty() || total < 2 * kPiece) {
            for (const CopyJob &j : jobs)
                memcpy(j.dst, j.src, j.bytes);
            return;
        }
        {
            /* a worker that woke late for the previous batch may still be
             * reading the piece list: rebuild it only when none is */
            std::unique_lock<std::mutex> lk(m_);
            idle_cv_.wait(lk, [this] { return active_ == 0; });
            pieces_.clear();
            for (const CopyJob &j : jobs)
                for (size_t o = 0; o < j.bytes; o += kPiece)
                    pieces_.push_back({ j.dst + o, j.src + o, std::min(kPiece, j.bytes - o) });
            next_.store(0, std::memory_order_relaxed);
            left_.store(pieces_.size(), std::memory_order_relaxed);
            gen_++;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> lk(m_);
        done_cv_.wait(lk, [this] { return left_.load(std::memory_order_acquire) == 0; });
    }

  private:
    void work()
    {
        const size_t n = pieces_.size();
        for (;;) {
            const size_t i = next_.fetch_add(1, std::memory_order_relaxed);
            if (i >= n)
                return;
            memcpy(pieces_[i].dst, pieces_[i].src, pieces_[i].bytes);
            if (left_.fetch_sub(1, std::memory_order_acq_rel) == 1) {
                std::lock_guard<std::mutex> lk(m_);
                done_cv_.notify_all();
            }
        }
    }

    void loop()
    {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_)
                    return;
                seen = gen_;
                active_++;
            }
            work();
            std::lock_guard<std::mutex> lk(m_);
            if (--active_ == 0)
                idle_cv_.notify_all();
        }
    }

    std::vector<std::thread> workers_;
    std::vector<CopyJob> pieces_;
    std::atomic<size_t> next_{ 0 };
    std::atomic<size_t> left_{ 0 };
    std::mutex m_;
    std::condition_variable cv_, done_cv_, idle_cv_;
    uint64_t gen_ = 0;
    int active_ = 0;   /* workers inside work() */
    bool stop_ = false;
};

} // namespace h261b
