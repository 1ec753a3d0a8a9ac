// ss_pool.hpp -- first-fit allocator over one device region, by offset.
//
// The serving loop admits a request only when its image and mask buffers fit
// in the device pool (admission by HBM footprint).  The pool hands out
// 256-byte aligned offsets into a region allocated once, so no device
// allocation happens while serving.  Free ranges are kept sorted by offset
// and merged with their neighbours on release.  Pure host code, no CUDA, so
// it is unit-tested on the CPU.
#pragma once

#include <cstddef>
#include <cstdint>
#include <iterator>
#include <map>

namespace ss {

class OffsetPool {
public:
    static constexpr size_t kAlign = 256;

    explicit OffsetPool(size_t capacity)
        : capacity_(capacity & ~(kAlign - 1)), free_total_(capacity_) {
        if (capacity_) {
            free_[0] = capacity_;
        }
    }

    static size_t round(size_t bytes) {
        return (bytes + kAlign - 1) & ~(kAlign - 1);
    }

    // First fit; false when no free range is large enough.
    bool alloc(size_t bytes, size_t* offset) {
        const size_t need = round(bytes == 0 ? 1 : bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= need) {
                const size_t off = it->first;
                const size_t rest = it->second - need;
                free_.erase(it);
                if (rest) {
                    free_[off + need] = rest;
                }
                free_total_ -= need;
                *offset = off;
                return true;
            }
        }
        return false;
    }

    // Returns a range given by alloc (same byte count).  False on a range
    // that overlaps free space or leaves the pool (a caller bug).
    bool release(size_t offset, size_t bytes) {
        const size_t size = round(bytes == 0 ? 1 : bytes);
        if (offset % kAlign || offset + size > capacity_ || offset + size < offset) {
            return false;
        }
        auto next = free_.lower_bound(offset);
        if (next != free_.end() && next->first < offset + size) {
            return false;
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second > offset) {
                return false;
            }
        }
        size_t start = offset;
        size_t len = size;
        if (next != free_.end() && next->first == offset + size) {
            len += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == offset) {
                start = prev->first;
                len += prev->second;
                free_.erase(prev);
            }
        }
        free_[start] = len;
        free_total_ += size;
        return true;
    }

    size_t capacity() const { return capacity_; }
    size_t free_bytes() const { return free_total_; }
    size_t used_bytes() const { return capacity_ - free_total_; }
    size_t free_ranges() const { return free_.size(); }
    size_t largest_free() const {
        size_t best = 0;
        for (const auto& kv : free_) {
            best = kv.second > best ? kv.second : best;
        }
        return best;
    }

private:
    size_t capacity_;
    size_t free_total_;
    std::map<size_t, size_t> free_;   // offset -> length
};

}  // namespace ss
