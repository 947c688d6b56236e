// Checks the host thread pool of simple-cpsd_b200/csrc/host_pool.h: jobs of
// random sizes, started and waited back to back (both entry points), each
// item must run exactly once.  Prints "ok" and exits 0, else the first
// failure and exits 1.  Built and run by tests/test_host.py.
#include <atomic>
#include <cstdio>
#include <random>
#include <vector>

#include "host_pool.h"

int main()
{
    auto &pool = cpsd_host::Pool::get();
    std::mt19937 rng(7);
    for (int it = 0; it < 5000; ++it) {
        const int n = (int)(rng() % 257);
        std::vector<std::atomic<int>> hit(n);
        for (auto &h : hit) h = 0;
        if (it & 1) {
            pool.run(n, [&](int i) { hit[i]++; });
        } else {
            pool.start(n, [&](int i) { hit[i]++; });
            pool.wait();
        }
        for (int i = 0; i < n; ++i)
            if (hit[i] != 1) {
                printf("job %d item %d ran %d times\n", it, i, (int)hit[i]);
                return 1;
            }
    }
    printf("ok %d threads\n", pool.threads());
    return 0;
}
