// First-fit allocator of the serving loop's device pool (abf_server.cpp):
// offsets into one range, no device calls, so it is also checked on the host
// alone (tests/pool_check.cpp).
#pragma once

#include <algorithm>
#include <cstdint>
#include <iterator>
#include <map>

namespace abf {

// First-fit allocator over one device range. Free extents are kept by
// offset and merged with their neighbours when a range comes back, so a
// pool whose results were all released is one extent again.
class Pool {
  public:
    static constexpr uint64_t kFail = ~0ull;
    void reset(uint64_t size) {
        free_.clear();
        if (size) free_[0] = size;
        used_ = 0;
    }
    uint64_t alloc(uint64_t n) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const uint64_t off = it->first, left = it->second - n;
            free_.erase(it);
            if (left) free_[off + n] = left;
            used_ += n;
            return off;
        }
        return kFail;
    }
    void release(uint64_t off, uint64_t n) {
        if (!n) return;
        used_ -= n;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + n == next->first) {
            n += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += n;
                return;
            }
        }
        free_[off] = n;
    }
    uint64_t largest() const {
        uint64_t m = 0;
        for (const auto& e : free_) m = std::max(m, e.second);
        return m;
    }
    uint64_t used() const { return used_; }
    const std::map<uint64_t, uint64_t>& free_extents() const { return free_; }

  private:
    std::map<uint64_t, uint64_t> free_;
    uint64_t used_ = 0;
};

}  // namespace abf
