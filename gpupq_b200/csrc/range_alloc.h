// First-fit allocator over an index range [0, size): the host-side bookkeeping behind the
// resident sessions' cell, tile and LP spaces.  Free ranges are kept sorted by start and
// merged with their neighbours when a range is returned.
#pragma once

#include <cstdint>
#include <iterator>
#include <map>
#include <utility>
#include <vector>

namespace gpq {

class RangeAlloc {
 public:
  void reset(uint64_t size) {
    free_.clear();
    if (size) free_[0] = size;
    size_ = size;
    used_ = 0;
  }
  // First free range that holds n; returns false (and changes nothing) when none does.
  bool alloc(uint64_t n, uint64_t* start) {
    if (n == 0) return false;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      *start = it->first;
      const uint64_t rest = it->second - n, next = it->first + n;
      free_.erase(it);
      if (rest) free_[next] = rest;
      used_ += n;
      return true;
    }
    return false;
  }
  void free(uint64_t start, uint64_t n) {
    if (n == 0) return;
    used_ -= n;
    auto next = free_.lower_bound(start);
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == start) {
        start = prev->first;
        n += prev->second;
        free_.erase(prev);
      }
    }
    if (next != free_.end() && start + n == next->first) {
      n += next->second;
      free_.erase(next);
    }
    free_[start] = n;
  }
  uint64_t used() const { return used_; }
  uint64_t size() const { return size_; }
  // The free ranges (start, length) in order, and the allocator set back to exactly them.
  std::vector<std::pair<uint64_t, uint64_t>> free_ranges() const { return {free_.begin(), free_.end()}; }
  void assign(uint64_t size, uint64_t used, const std::vector<std::pair<uint64_t, uint64_t>>& ranges) {
    free_.clear();
    for (const auto& r : ranges) free_[r.first] = r.second;
    size_ = size;
    used_ = used;
  }

 private:
  std::map<uint64_t, uint64_t> free_;  // start -> length
  uint64_t size_ = 0, used_ = 0;
};

}  // namespace gpq
