// Randomised check of the serving pool's first-fit allocator: no two live
// ranges overlap, accounting matches, releases merge back to one range.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "ss_pool.hpp"

struct Live {
    size_t off, bytes;
};

static int fail(const char* what, int step) {
    std::printf("FAIL %s at step %d\n", what, step);
    return 1;
}

int main() {
    const size_t cap = (64u << 20) + 100;   // not a multiple of 256
    ss::OffsetPool pool(cap);
    if (pool.capacity() != (64u << 20)) return fail("capacity rounding", 0);
    std::mt19937_64 rng(12345);
    std::vector<Live> live;
    size_t used = 0;
    for (int step = 0; step < 200000; ++step) {
        const bool do_alloc = live.empty() || (rng() % 100) < 55;
        if (do_alloc) {
            size_t bytes = 1 + rng() % (3u << 20);
            if (rng() % 10 == 0) bytes = 1 + rng() % 512;
            size_t off = 0;
            if (pool.alloc(bytes, &off)) {
                const size_t r = ss::OffsetPool::round(bytes);
                if (off % 256) return fail("alignment", step);
                if (off + r > pool.capacity()) return fail("bounds", step);
                for (const Live& l : live) {
                    const size_t lr = ss::OffsetPool::round(l.bytes);
                    if (off < l.off + lr && l.off < off + r)
                        return fail("overlap", step);
                }
                live.push_back({off, bytes});
                used += r;
            } else if (pool.largest_free() >= ss::OffsetPool::round(bytes)) {
                return fail("first fit missed a large enough range", step);
            }
        } else {
            const size_t k = rng() % live.size();
            if (!pool.release(live[k].off, live[k].bytes))
                return fail("release", step);
            used -= ss::OffsetPool::round(live[k].bytes);
            live[k] = live.back();
            live.pop_back();
        }
        if (pool.used_bytes() != used) return fail("accounting", step);
    }
    // A range that is already free, or leaves the pool, is refused.
    size_t off = 0;
    for (const Live& l : live) pool.release(l.off, l.bytes);
    if (pool.free_ranges() != 1 || pool.free_bytes() != pool.capacity())
        return fail("merge", 0);
    if (pool.release(0, 256)) return fail("double release", 0);
    if (pool.release(pool.capacity(), 256)) return fail("out of range", 0);
    if (!pool.alloc(pool.capacity(), &off) || off != 0)
        return fail("whole pool", 0);
    if (pool.alloc(1, &off)) return fail("full pool", 0);
    std::printf("OK\n");
    return 0;
}
