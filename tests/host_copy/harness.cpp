// Host-copy pool check (hype-parallel_b200/csrc/hype_hostcopy.cu), no GPU needed:
// contiguous and pitched copies of assorted sizes equal memcpy's result; copies
// issued from several threads at once (the pool takes one at a time) are all
// correct; a forked child gets a pool of its own and copies correctly.  Prints
// "ok" and exits 0, or names the first failure and exits 1.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <thread>
#include <vector>
#include <sys/wait.h>
#include <unistd.h>

namespace hype {
void host_copy(void *dst, const void *src, size_t bytes);
void host_copy_2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width, size_t rows);
}

static bool check_contiguous(std::mt19937_64 &rng, size_t bytes)
{
    std::vector<unsigned char> a(bytes + 64), b(bytes + 64, 0xAB);
    for (auto &x : a) x = (unsigned char)rng();
    const size_t off = rng() % (bytes < 16 ? bytes : 16);   // unaligned starts too
    hype::host_copy(b.data() + off, a.data() + off, bytes - off);
    if (std::memcmp(b.data() + off, a.data() + off, bytes - off) != 0) return false;
    for (size_t k = 0; k < off; ++k)
        if (b[k] != 0xAB) return false;   // nothing written before the destination
    for (size_t k = bytes; k < b.size(); ++k)
        if (b[k] != 0xAB) return false;   // nor after it
    return true;
}

static bool check_pitched(std::mt19937_64 &rng, size_t width, size_t rows, size_t spitch, size_t dpitch)
{
    std::vector<unsigned char> a(spitch * rows), b(dpitch * rows, 0xCD);
    for (auto &x : a) x = (unsigned char)rng();
    hype::host_copy_2d(b.data(), dpitch, a.data(), spitch, width, rows);
    for (size_t r = 0; r < rows; ++r) {
        if (std::memcmp(b.data() + r * dpitch, a.data() + r * spitch, width) != 0) return false;
        for (size_t k = width; k < dpitch; ++k)
            if (b[r * dpitch + k] != 0xCD) return false;   // the gaps between rows stay untouched
    }
    return true;
}

int main()
{
    std::mt19937_64 rng(7);
    const size_t sizes[] = {1, 15, 4096, 65536, 65537, (1u << 20) - 3, (5u << 20) + 11, 37u << 20};
    for (size_t n : sizes)
        if (!check_contiguous(rng, n)) { std::printf("contiguous copy of %zu bytes differs\n", n); return 1; }
    struct P { size_t w, rows, sp, dp; };
    const P pitched[] = {{48, 1, 48, 48}, {1000, 37, 1048, 1000}, {49152, 700, 49440, 49152}, {98304, 300, 98592, 98400}, {7, 5000, 13, 9}};
    for (const P &q : pitched)
        if (!check_pitched(rng, q.w, q.rows, q.sp, q.dp)) { std::printf("pitched copy %zu x %zu differs\n", q.w, q.rows); return 1; }
    // several threads at once
    std::vector<std::thread> th;
    std::vector<int> ok(6, 0);
    for (int t = 0; t < 6; ++t)
        th.emplace_back([&, t] {
            std::mt19937_64 r(100 + t);
            bool good = true;
            for (int k = 0; k < 20 && good; ++k) good = check_contiguous(r, (size_t)(r() % (3u << 20)) + 16);
            ok[t] = good;
        });
    for (auto &x : th) x.join();
    for (int t = 0; t < 6; ++t)
        if (!ok[t]) { std::printf("concurrent copies of thread %d differ\n", t); return 1; }
    // a forked child: its own pool
    const pid_t pid = fork();
    if (pid == 0) {
        std::mt19937_64 r(9);
        _exit(check_contiguous(r, 3u << 20) && check_pitched(r, 1000, 37, 1048, 1000) ? 0 : 3);
    }
    int status = 0;
    if (pid < 0 || waitpid(pid, &status, 0) != pid || !WIFEXITED(status) || WEXITSTATUS(status) != 0) {
        std::printf("copy in a forked child failed (status %d)\n", status);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
