// hype_hostcopy.cu -- host-side copies between a caller's pageable arrays and the
// solver's pinned staging buffers, split over a small thread pool.
//
// The host calls (hype_rhs_prim, hype_rhs_prim_slab, hype_advance_host) stream a
// state through the GPU in row bands.  From pinned memory the copy engines move
// 54-56 GB/s each way; from pageable memory (PETSc's Vec arrays, numpy arrays)
// the driver stages each copy itself at 11 GB/s up and 17.5 GB/s down on a B200
// host, while four threads copy pageable to pinned memory at about 46 GB/s.  So
// a pageable band is copied into pinned staging by the pool, and the copy
// engine takes it from there (and the reverse on the way out).
#include "hype_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <unistd.h>

namespace hype {
namespace {

// One 2-D copy at a time (rows of `width` bytes, `dpitch` / `spitch` apart),
// split into row blocks that the workers and the calling thread take in turn.
// A worker takes a snapshot of the task and registers as active under the lock;
// the caller starts a task only while no worker is active and returns only once
// every part is done and no worker is active, so no worker ever reads a task
// that changes under it or touches memory after the copy has returned.
struct CopyPool {
    static constexpr int WORKERS = 3;   // + the caller: 4 threads, the measured best
    struct Task {
        char *dst = nullptr;
        const char *src = nullptr;
        size_t dpitch = 0, spitch = 0, width = 0, rows = 0, rows_per_part = 0;
        int parts = 0;
    };
    std::mutex call_m;   // one copy at a time
    std::mutex m;
    std::condition_variable cv, done_cv;
    unsigned long long gen = 0;
    Task task;
    int active = 0;
    std::atomic<int> next{0};
    std::atomic<int> remaining{0};
    pid_t pid = getpid();

    CopyPool()
    {
        for (int k = 0; k < WORKERS; ++k) std::thread([this] { work(); }).detach();
    }

    void run_parts(const Task &t)
    {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= t.parts) return;
            const size_t r0 = (size_t)i * t.rows_per_part, r1 = std::min(t.rows, r0 + t.rows_per_part);
            if (t.dpitch == t.width && t.spitch == t.width)
                std::memcpy(t.dst + r0 * t.width, t.src + r0 * t.width, (r1 - r0) * t.width);
            else
                for (size_t r = r0; r < r1; ++r) std::memcpy(t.dst + r * t.dpitch, t.src + r * t.spitch, t.width);
            if (remaining.fetch_sub(1) == 1) {
                std::lock_guard<std::mutex> g(m);
                done_cv.notify_all();
            }
        }
    }

    void work()
    {
        unsigned long long seen = 0;
        for (;;) {
            Task t;
            {
                std::unique_lock<std::mutex> lk(m);
                cv.wait(lk, [&] { return gen != seen; });
                seen = gen;
                t = task;
                ++active;
            }
            run_parts(t);
            std::lock_guard<std::mutex> g(m);
            --active;
            done_cv.notify_all();
        }
    }

    void copy(void *d, size_t dp, const void *s, size_t sp, size_t w, size_t nrows)
    {
        if (!w || !nrows) return;
        std::lock_guard<std::mutex> call(call_m);
        const size_t bytes = w * nrows;
        const size_t want = std::min<size_t>(4 * (WORKERS + 1), std::max<size_t>(1, bytes >> 20));   // >= 1 MiB a part
        Task t;
        t.dst = (char *)d; t.src = (const char *)s;
        t.dpitch = dp; t.spitch = sp; t.width = w; t.rows = nrows;
        t.rows_per_part = (nrows + want - 1) / want;
        t.parts = (int)((nrows + t.rows_per_part - 1) / t.rows_per_part);
        {
            std::unique_lock<std::mutex> lk(m);
            done_cv.wait(lk, [&] { return active == 0; });   // a straggler of the last copy
            task = t;
            remaining.store(t.parts);
            next.store(0);
            ++gen;
        }
        cv.notify_all();
        run_parts(t);   // the caller takes parts too, so the copy finishes even without workers
        std::unique_lock<std::mutex> lk(m);
        done_cv.wait(lk, [&] { return remaining.load() == 0 && active == 0; });
    }
};

CopyPool *pool()
{
    // one pool per process; a forked child (whose copy has no worker threads and
    // may hold a locked mutex) starts a pool of its own.  Never destroyed: its
    // detached workers wait on it until the process ends.
    static std::mutex m;
    static CopyPool *p = nullptr;
    std::lock_guard<std::mutex> g(m);
    if (!p || p->pid != getpid()) p = new CopyPool();
    return p;
}

}  // namespace

void host_copy_2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width, size_t rows)
{
    pool()->copy(dst, dpitch, src, spitch, width, rows);
}

void host_copy(void *dst, const void *src, size_t bytes)
{
    // as rows of 64 KiB (and one row for the rest), so that the parts split it
    constexpr size_t W = 64 << 10;
    const size_t rows = bytes / W, tail = bytes - rows * W;
    if (rows) pool()->copy(dst, W, src, W, W, rows);
    if (tail) std::memcpy((char *)dst + rows * W, (const char *)src + rows * W, tail);
}

bool host_is_pageable(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();   // older drivers report unregistered memory as an error
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

}  // namespace hype
