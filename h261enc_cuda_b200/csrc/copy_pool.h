/* Host copy workers for the staging arena.
 *
 * A batch of pictures submitted in one call is copied into the pinned
 * staging arena by a small persistent pool: every plane copy is cut into
 * pieces of at most kPiece bytes, the pieces are taken from one atomic
 * counter by the workers and by the calling thread, and the call returns
 * when the last piece is done.  A batch started without waiting is
 * finished by the workers and by whichever thread joins it (the next
 * step).  Workers sleep on a condition variable between batches. */
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <system_error>
#include <thread>
#include <vector>

#if defined(__x86_64__) || defined(__SSE2__)
#include <emmintrin.h>
#define H261B_STREAM_STORES 1
#endif

namespace h261b {

/* memcpy into pinned memory that the device reads next: streaming stores
 * write the destination without first reading it into the cache (a third
 * less memory traffic than a plain copy, and none of it left in the cache
 * that the DMA engine would then have to snoop).  The caller fences. */
inline void stream_copy(uint8_t *dst, const uint8_t *src, size_t n)
{
#ifdef H261B_STREAM_STORES
    size_t head = (16 - ((uintptr_t)dst & 15)) & 15;
    if (head > n)
        head = n;
    memcpy(dst, src, head);
    dst += head;
    src += head;
    n -= head;
    size_t i = 0;
    for (; i + 64 <= n; i += 64) {
        const __m128i a = _mm_loadu_si128((const __m128i *)(src + i));
        const __m128i b = _mm_loadu_si128((const __m128i *)(src + i + 16));
        const __m128i c = _mm_loadu_si128((const __m128i *)(src + i + 32));
        const __m128i d = _mm_loadu_si128((const __m128i *)(src + i + 48));
        _mm_stream_si128((__m128i *)(dst + i), a);
        _mm_stream_si128((__m128i *)(dst + i + 16), b);
        _mm_stream_si128((__m128i *)(dst + i + 32), c);
        _mm_stream_si128((__m128i *)(dst + i + 48), d);
    }
    memcpy(dst + i, src + i, n - i);
#else
    memcpy(dst, src, n);
#endif
}

inline void stream_fence()
{
#ifdef H261B_STREAM_STORES
    _mm_sfence();
#endif
}

struct CopyJob {
    uint8_t *dst;
    const uint8_t *src;
    size_t bytes;
};

class CopyPool {
  public:
    static constexpr size_t kPiece = 64 << 10;

    /* Starts up to `threads` workers.  A worker the system cannot start
     * (std::system_error from thread creation) is left out: the pool runs
     * with the ones that started, down to none, in which case the calling
     * thread copies every batch itself.  `spawn` creates a worker thread
     * (tests pass one that fails); `on_piece`, when set, runs in a worker
     * before each piece it copies (tests stall a worker with it). */
    using Spawn = std::function<std::thread(std::function<void()>)>;
    explicit CopyPool(int threads, Spawn spawn = nullptr, std::function<void(int)> on_piece = nullptr)
        : on_piece_(std::move(on_piece))
    {
        if (!spawn)
            spawn = [](std::function<void()> f) { return std::thread(std::move(f)); };
        for (int i = 0; i < threads; i++) {
            try {
                workers_.push_back(spawn([this, i] { loop(i); }));
            } catch (const std::system_error &) {
                break;
            }
        }
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
        join();
        size_t total = 0;
        for (const CopyJob &j : jobs)
            total += j.bytes;
        if (workers_.empty() || total < 2 * kPiece) {
            for (const CopyJob &j : jobs)
                stream_copy(j.dst, j.src, j.bytes);
            stream_fence();
            return;
        }
        publish(jobs);
        work();
        join();
    }

    /* start copying every job on the workers and return at once; join()
     * (or the next run / start) waits for the bytes */
    void start(const std::vector<CopyJob> &jobs)
    {
        join();
        if (workers_.empty()) {
            for (const CopyJob &j : jobs)
                stream_copy(j.dst, j.src, j.bytes);
            stream_fence();
            return;
        }
        publish(jobs);
    }

    /* wait until the batch in flight (if any) is copied; the caller takes
     * pieces of it meanwhile instead of only waiting */
    void join()
    {
        if (left_.load(std::memory_order_acquire) != 0)
            work();
        std::unique_lock<std::mutex> lk(m_);
        done_cv_.wait(lk, [this] { return left_.load(std::memory_order_acquire) == 0; });
    }

    bool busy() const { return left_.load(std::memory_order_acquire) != 0; }

  private:
    void publish(const std::vector<CopyJob> &jobs)
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
        lk.unlock();
        cv_.notify_all();
    }

    /* copy pieces until none is left; worker = -1 for a calling thread */
    void work(int worker = -1)
    {
        const size_t n = pieces_.size();
        for (;;) {
            const size_t i = next_.fetch_add(1, std::memory_order_relaxed);
            if (i >= n)
                return;
            if (worker >= 0 && on_piece_)
                on_piece_(worker);
            stream_copy(pieces_[i].dst, pieces_[i].src, pieces_[i].bytes);
            stream_fence();   /* visible before the batch counts as done */
            if (left_.fetch_sub(1, std::memory_order_acq_rel) == 1) {
                std::lock_guard<std::mutex> lk(m_);
                done_cv_.notify_all();
            }
        }
    }

    void loop(int worker)
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
            work(worker);
            std::lock_guard<std::mutex> lk(m_);
            if (--active_ == 0)
                idle_cv_.notify_all();
        }
    }

    std::function<void(int)> on_piece_;
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
