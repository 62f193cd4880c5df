// serve_sched.h — host-side bookkeeping of the sampling server (no CUDA).
//
// Arena: first-fit allocator of request buffers inside one device region;
// requests are admitted by their HBM footprint (f rows + output rows), so the
// arena's size is the admission budget.  admissible(): requests are admitted
// strictly in arrival order; the head waits until the arena, a request slot,
// enough job slots and ring room are all free (no bypass, so a large request
// is never starved by a stream of small ones).  All of it is plain C++, so it
// is unit-tested on the CPU.
#pragma once
#include <stdint.h>

#include <iterator>
#include <map>
#include <vector>

namespace ksim {

class Arena {
public:
    explicit Arena(int64_t capacity = 0, int64_t align = 256) { reset(capacity, align); }

    void reset(int64_t capacity, int64_t align = 256)
    {
        cap_ = capacity < 0 ? 0 : capacity;
        align_ = align <= 0 ? 1 : align;
        free_.clear();
        used_.clear();
        in_use_ = 0;
        if (cap_ > 0) free_[0] = cap_;
    }

    static int64_t round_up(int64_t n, int64_t a) { return (n + a - 1) / a * a; }

    // Offset of a block of at least `bytes` (>= 1), or -1 when no free block fits.
    int64_t alloc(int64_t bytes)
    {
        const int64_t need = round_up(bytes < 1 ? 1 : bytes, align_);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < need) continue;
            const int64_t off = it->first, size = it->second;
            free_.erase(it);
            if (size > need) free_[off + need] = size - need;
            used_[off] = need;
            in_use_ += need;
            return off;
        }
        return -1;
    }

    // Return a block; adjacent free blocks are merged.  False if `off` is not
    // the start of a live block.
    bool release(int64_t off)
    {
        auto u = used_.find(off);
        if (u == used_.end()) return false;
        int64_t start = off, size = u->second;
        in_use_ -= size;
        used_.erase(u);
        auto next = free_.lower_bound(start);
        if (next != free_.end() && next->first == start + size) {
            size += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == start) {
                start = prev->first;
                size += prev->second;
                free_.erase(prev);
            }
        }
        free_[start] = size;
        return true;
    }

    int64_t capacity() const { return cap_; }
    int64_t align() const { return align_; }
    int64_t in_use() const { return in_use_; }
    int64_t largest_free() const
    {
        int64_t m = 0;
        for (const auto &kv : free_) m = kv.second > m ? kv.second : m;
        return m;
    }
    int64_t free_blocks() const { return (int64_t)free_.size(); }
    int64_t live_blocks() const { return (int64_t)used_.size(); }
    // A request of `bytes` could be admitted into an empty arena.
    bool ever_fits(int64_t bytes) const { return round_up(bytes < 1 ? 1 : bytes, align_) <= cap_; }

private:
    int64_t cap_ = 0, align_ = 256, in_use_ = 0;
    std::map<int64_t, int64_t> free_;  // offset -> size
    std::map<int64_t, int64_t> used_;  // offset -> size
};

// A LIFO pool of integer slots [0, n).
class SlotPool {
public:
    explicit SlotPool(int n = 0) { reset(n); }
    void reset(int n)
    {
        free_.clear();
        for (int i = n - 1; i >= 0; --i) free_.push_back(i);
        n_ = n;
    }
    int take()
    {
        if (free_.empty()) return -1;
        const int s = free_.back();
        free_.pop_back();
        return s;
    }
    void give(int s) { free_.push_back(s); }
    int available() const { return (int)free_.size(); }
    int size() const { return n_; }

private:
    std::vector<int> free_;
    int n_ = 0;
};

// What admitting the head request needs, and whether it is available now.
struct AdmitNeed {
    int64_t bytes;     // arena bytes (f rows + output rows)
    int jobs;          // job-table slots (components with outputs)
    int64_t ring;      // ring entries (one per job)
};

struct AdmitState {
    Arena *arena;
    SlotPool *req_slots, *job_slots;
    int64_t ring_cap, ring_in_flight;
};

// 1: admissible now; 0: must wait for resources to free up; -1: can never
// be admitted (larger than the whole arena, job table or ring).
inline int admissible(const AdmitNeed &n, const AdmitState &s)
{
    if (!s.arena->ever_fits(n.bytes) || n.jobs > s.job_slots->size() || n.ring > s.ring_cap) return -1;
    if (s.req_slots->available() < 1 || s.job_slots->available() < n.jobs) return 0;
    if (s.ring_in_flight + n.ring > s.ring_cap) return 0;
    return s.arena->largest_free() >= Arena::round_up(n.bytes < 1 ? 1 : n.bytes, s.arena->align()) ? 1 : 0;
}

}  // namespace ksim
