// First-fit sub-allocator over one fixed range of device memory (host-side bookkeeping only).
// The serving loop reserves its whole memory budget once and places each admitted request's
// projections, workspace and volume in one block of it, so admission is a bookkeeping decision
// and no device allocation happens while requests run. Free blocks are kept sorted by offset and
// coalesced with their neighbours on release.
#pragma once

#include <cstddef>
#include <cstdint>
#include <iterator>
#include <map>

namespace gct {

class Arena {
public:
    static constexpr size_t kAlign = 256;

    explicit Arena(size_t bytes = 0) { reset(bytes); }

    void reset(size_t bytes)
    {
        free_.clear();
        used_.clear();
        size_ = bytes & ~(kAlign - 1);
        in_use_ = peak_ = 0;
        if (size_) free_[0] = size_;
    }

    static size_t round_up(size_t n) { return (n + kAlign - 1) & ~(kAlign - 1); }

    // Offset of a block of at least n bytes (kAlign-aligned), or SIZE_MAX if no free block fits.
    size_t alloc(size_t n)
    {
        n = round_up(n == 0 ? 1 : n);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const size_t off = it->first, rest = it->second - n;
            free_.erase(it);
            if (rest) free_[off + n] = rest;
            used_[off] = n;
            in_use_ += n;
            if (in_use_ > peak_) peak_ = in_use_;
            return off;
        }
        return SIZE_MAX;
    }

    // Releases the block at off; false if off is not the start of a live block.
    bool release(size_t off)
    {
        auto u = used_.find(off);
        if (u == used_.end()) return false;
        size_t start = off, len = u->second;
        used_.erase(u);
        in_use_ -= len;
        auto next = free_.lower_bound(start);
        if (next != free_.end() && start + len == next->first) {
            len += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == start) {
                start = prev->first;
                len += prev->second;
                free_.erase(prev);
            }
        }
        free_[start] = len;
        return true;
    }

    bool fits(size_t n) const
    {
        n = round_up(n == 0 ? 1 : n);
        for (const auto &f : free_)
            if (f.second >= n) return true;
        return false;
    }

    size_t size() const { return size_; }
    size_t in_use() const { return in_use_; }
    size_t peak() const { return peak_; }
    size_t free_blocks() const { return free_.size(); }
    size_t live_blocks() const { return used_.size(); }

private:
    std::map<size_t, size_t> free_;  // offset -> length
    std::map<size_t, size_t> used_;  // offset -> length
    size_t size_ = 0, in_use_ = 0, peak_ = 0;
};

}  // namespace gct
