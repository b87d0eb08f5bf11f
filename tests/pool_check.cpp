// Host-side check of the serving loop's pool allocator (abf_pool.h): random
// allocations, whole and partial releases (the server trims a batch's id
// room and frees its bitmaps separately), against a shadow list of live
// ranges. After every step: live ranges lie inside the pool and do not
// overlap, free extents are sorted, disjoint, merged with their neighbours
// and disjoint from live ranges, and free + used bytes add up to the pool.
// Once everything is released the pool is one extent again.
#include "abf_pool.h"

#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

namespace {
struct Range {
    uint64_t off, n;
};

int fail(const char* what, int step) {
    std::printf("FAIL at step %d: %s\n", step, what);
    return 1;
}

int check(const abf::Pool& p, const std::vector<Range>& live, uint64_t size, int step) {
    uint64_t used = 0;
    std::vector<Range> all = live;
    for (const Range& r : live) {
        if (r.off + r.n > size) return fail("live range outside the pool", step);
        used += r.n;
    }
    if (used != p.used()) return fail("used bytes", step);
    uint64_t free_bytes = 0, prev_end = 0;
    bool first = true;
    for (const auto& e : p.free_extents()) {
        if (e.second == 0) return fail("empty free extent", step);
        if (!first && e.first < prev_end) return fail("free extents overlap", step);
        if (!first && e.first == prev_end) return fail("adjacent free extents not merged", step);
        if (e.first + e.second > size) return fail("free extent outside the pool", step);
        prev_end = e.first + e.second;
        first = false;
        free_bytes += e.second;
        all.push_back({e.first, e.second});
    }
    if (free_bytes + used != size) return fail("free + used != pool", step);
    // every byte is in exactly one range: sorted, no overlap, no gap
    std::sort(all.begin(), all.end(), [](const Range& a, const Range& b) { return a.off < b.off; });
    uint64_t at = 0;
    for (const Range& r : all) {
        if (r.off != at) return fail("ranges overlap or leave a gap", step);
        at += r.n;
    }
    if (at != size) return fail("ranges do not cover the pool", step);
    return 0;
}
}  // namespace

int main() {
    const uint64_t size = 1ull << 30;
    std::mt19937_64 rng(12345);
    for (int round = 0; round < 4; ++round) {
        abf::Pool p;
        p.reset(size);
        std::vector<Range> live;
        int step = 0;
        for (; step < 20000; ++step) {
            const int op = int(rng() % 10);
            if (op < 5 || live.empty()) {  // allocate 256 B .. 8 MB in 256-byte units
                const uint64_t n = (1 + rng() % 32768) * 256;
                const uint64_t off = p.alloc(n);
                if (off == abf::Pool::kFail) {
                    if (p.largest() >= n) return fail("alloc failed with room", step);
                } else {
                    live.push_back({off, n});
                }
            } else if (op < 8) {  // release a whole range
                const size_t i = rng() % live.size();
                p.release(live[i].off, live[i].n);
                live.erase(live.begin() + long(i));
            } else {  // release the tail or the head of a range, keep the rest
                const size_t i = rng() % live.size();
                Range& r = live[i];
                if (r.n < 512) continue;
                const uint64_t cut = (1 + rng() % (r.n / 256 - 1)) * 256;
                if (op == 8) {
                    p.release(r.off + cut, r.n - cut);
                    r.n = cut;
                } else {
                    p.release(r.off, cut);
                    r.off += cut;
                    r.n -= cut;
                }
            }
            if (check(p, live, size, step)) return 1;
        }
        for (const Range& r : live) p.release(r.off, r.n);
        live.clear();
        if (check(p, live, size, step)) return 1;
        if (p.free_extents().size() != 1 || p.largest() != size) return fail("pool not one extent at the end", step);
    }
    std::printf("ok\n");
    return 0;
}
