// range_alloc.h — first-fit allocator of offsets in a fixed range (the
// device arenas of the batched form and of the serving loop's solo slots:
// allocated once, then carved without cudaMalloc).
#pragma once

#include <iterator>
#include <map>

namespace dimgpu {

// First-fit allocator of ranges of [0, capacity): the arena mode's cells and
// dt-log entries.  Freed ranges merge with their neighbours.
class RangeAlloc {
public:
    void reset(long long cap)
    {
        free_.clear();
        if (cap > 0) free_[0] = cap;
        used_ = 0;
    }
    long long alloc(long long n)
    {
        if (n <= 0) n = 1;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const long long off = it->first, len = it->second;
            free_.erase(it);
            if (len > n) free_[off + n] = len - n;
            used_ += n;
            return off;
        }
        return -1;
    }
    void release(long long off, long long n)
    {
        if (n <= 0) n = 1;
        used_ -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    long long used() const { return used_; }

private:
    std::map<long long, long long> free_;
    long long used_ = 0;
};

}  // namespace dimgpu
