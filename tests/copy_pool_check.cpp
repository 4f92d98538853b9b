// Host-side check of the staging copy pool (h261enc_cuda_b200/csrc/copy_pool.h):
// batches of plane copies cut into pieces, copied by the workers and by the
// caller of run(); start() returns at once and the next start, run or join
// waits for that batch.  Built and run by tests/test_copy_pool.py; prints "ok"
// and exits 0 on success.
#include "copy_pool.h"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <system_error>
#include <thread>
#include <vector>

using h261b::CopyJob;
using h261b::CopyPool;

static int fail(const char *what, long a = 0, long b = 0)
{
    std::printf("FAIL %s %ld %ld\n", what, a, b);
    return 1;
}

/* one batch: `planes` copies of random sizes from src into dst at random offsets */
struct Batch {
    std::vector<uint8_t> src, dst;
    std::vector<CopyJob> jobs;
};

static void make_batch(Batch &b, std::mt19937 &rng, int planes)
{
    size_t total = 0;
    std::vector<size_t> sizes, gaps;
    for (int i = 0; i < planes; i++) {
        sizes.push_back(1 + rng() % (300 << 10));   /* up to several pieces each */
        gaps.push_back(rng() % 64);
        total += sizes.back() + gaps.back();
    }
    b.src.resize(total);
    b.dst.assign(total, 0);
    for (auto &x : b.src)
        x = (uint8_t)(rng() | 1);
    size_t o = 0;
    for (int i = 0; i < planes; i++) {
        b.jobs.push_back({ b.dst.data() + o, b.src.data() + o, sizes[i] });
        o += sizes[i] + gaps[i];
    }
}

static bool landed(const Batch &b)
{
    for (const CopyJob &j : b.jobs)
        if (std::memcmp(j.dst, j.src, j.bytes) != 0)
            return false;
    return true;
}

int main()
{
    std::mt19937 rng(2026);
    for (int workers : { 0, 1, 3, 7 }) {
        CopyPool pool(workers);
        std::vector<Batch> batches(24);
        for (size_t i = 0; i < batches.size(); i++) {
            make_batch(batches[i], rng, 1 + (int)(rng() % 12));
            if (i % 3 == 2) {
                /* synchronous: in place on return, and so is the batch
                 * started before it */
                pool.run(batches[i].jobs);
                for (size_t k = 0; k <= i; k++)
                    if (!landed(batches[k]))
                        return fail("run returned before a batch landed", workers, (long)k);
            } else {
                /* asynchronous: the next start, run or join waits for it */
                pool.start(batches[i].jobs);
                if (i % 3 == 1) {
                    pool.join();
                    if (pool.busy())
                        return fail("busy after join", workers, (long)i);
                    for (size_t k = 0; k <= i; k++)
                        if (!landed(batches[k]))
                            return fail("join returned before a batch landed", workers, (long)k);
                }
            }
        }
        pool.join();
        /* an empty batch completes at once */
        const std::vector<CopyJob> none;
        pool.start(none);
        pool.join();
        if (pool.busy())
            return fail("busy after an empty batch", workers);
    }
    /* failures injected on the host: workers that cannot be started, and
     * a worker that stalls in the middle of a batch */
    for (int started : { 0, 2 }) {
        /* thread creation fails after `started` workers (resource
         * exhaustion): the pool keeps those and every batch still lands */
        int made = 0;
        CopyPool pool(6, [&](std::function<void()> f) {
            if (made == started)
                throw std::system_error(std::make_error_code(std::errc::resource_unavailable_try_again));
            made++;
            return std::thread(std::move(f));
        });
        if (pool.threads() != started)
            return fail("workers after a failed start", started, pool.threads());
        for (int i = 0; i < 6; i++) {
            Batch b;
            make_batch(b, rng, 8);
            if (i % 2)
                pool.run(b.jobs);
            else {
                pool.start(b.jobs);
                pool.join();
            }
            if (!landed(b))
                return fail("a batch did not land with workers missing", started, i);
        }
    }
    {
        /* worker 0 sleeps before each piece: the caller and the other
         * workers take the rest, and run / join still return only once
         * every byte is in place */
        std::atomic<int> stalls{ 0 };
        CopyPool pool(3, nullptr, [&](int w) {
            if (w == 0) {
                stalls++;
                std::this_thread::sleep_for(std::chrono::milliseconds(20));
            }
        });
        for (int i = 0; i < 6; i++) {
            Batch b;
            make_batch(b, rng, 12);
            if (i % 2)
                pool.run(b.jobs);
            else {
                pool.start(b.jobs);
                pool.join();
            }
            if (!landed(b) || pool.busy())
                return fail("a batch did not land around a stalled worker", i);
        }
        if (stalls.load() == 0)
            return fail("the stalled worker never took a piece");
    }
    std::printf("ok\n");
    return 0;
}
