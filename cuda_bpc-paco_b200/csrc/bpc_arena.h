// bpc_arena.h -- first-fit allocator over the address-ordered free ranges of
// one preallocated region (the request server's device-memory budget).  Pure
// host code: offsets and sizes only, no device calls.
#pragma once
#include <cstddef>
#include <iterator>
#include <map>

namespace bpc {

class Arena {
   public:
    void init(size_t n) {
        free_.clear();
        free_[0] = n;
        used_ = 0;
    }
    // lowest-addressed free range that fits n bytes; false if none does
    bool alloc(size_t n, size_t *off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            *off = it->first;
            const size_t rest = it->second - n, at = it->first + n;
            free_.erase(it);
            if (rest) free_[at] = rest;
            used_ += n;
            return true;
        }
        return false;
    }
    // give [off, off + n) back, merging with free neighbours
    void release(size_t off, size_t n) {
        used_ -= n;
        auto nx = free_.lower_bound(off);
        if (nx != free_.end() && off + n == nx->first) {  // merge with the next range
            n += nx->second;
            nx = free_.erase(nx);
        }
        if (nx != free_.begin()) {  // merge with the previous range
            auto pv = std::prev(nx);
            if (pv->first + pv->second == off) {
                pv->second += n;
                return;
            }
        }
        free_[off] = n;
    }
    size_t used() const { return used_; }
    size_t free_ranges() const { return free_.size(); }
    size_t largest_free() const {
        size_t m = 0;
        for (const auto &kv : free_) m = kv.second > m ? kv.second : m;
        return m;
    }

   private:
    std::map<size_t, size_t> free_;  // offset -> length
    size_t used_ = 0;
};

}  // namespace bpc
