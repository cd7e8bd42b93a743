// elmm_arena.h -- first-fit sub-allocator over one device allocation: the HBM
// budget of the serving loop.  Admission of a request is an allocation from
// its arena; a finished request returns its extents, and neighbouring free
// extents merge.  Plain host bookkeeping over offsets (no CUDA calls), so the
// device memory it hands out is never allocated or freed while kernels run.
#pragma once

#include <cstddef>
#include <cstdint>
#include <iterator>
#include <map>

namespace elmm {

class Arena {
 public:
  static constexpr size_t kAlign = 256;

  Arena() = default;
  Arena(char *base, size_t size) { reset(base, size); }

  void reset(char *base, size_t size) {
    base_ = base;
    size_ = size / kAlign * kAlign;
    free_.clear();
    used_.clear();
    if (size_) free_[0] = size_;
    in_use_ = 0;
    peak_ = 0;
  }

  // first free extent that holds `bytes` (rounded up to kAlign), or nullptr
  char *alloc(size_t bytes) {
    const size_t need = round(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < need) continue;
      const size_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > need) free_[off + need] = len - need;
      used_[off] = need;
      in_use_ += need;
      if (in_use_ > peak_) peak_ = in_use_;
      return base_ + off;
    }
    return nullptr;
  }

  // returns an extent of alloc(); false for a pointer it did not hand out
  bool release(const void *p) {
    if (!p) return true;
    const size_t off = (size_t)((const char *)p - base_);
    auto u = used_.find(off);
    if ((const char *)p < base_ || u == used_.end()) return false;
    size_t start = off, len = u->second;
    used_.erase(u);
    in_use_ -= len;
    auto next = free_.lower_bound(start);
    if (next != free_.end() && next->first == start + len) {  // merge with the extent after
      len += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {  // merge with the extent before
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

  size_t capacity() const { return size_; }
  size_t in_use() const { return in_use_; }
  size_t peak() const { return peak_; }
  size_t largest_free() const {
    size_t m = 0;
    for (auto &e : free_)
      if (e.second > m) m = e.second;
    return m;
  }
  size_t free_extents() const { return free_.size(); }
  bool empty() const { return used_.empty(); }
  static size_t round(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

 private:
  char *base_ = nullptr;
  size_t size_ = 0, in_use_ = 0, peak_ = 0;
  std::map<size_t, size_t> free_;  // offset -> length
  std::map<size_t, size_t> used_;  // offset -> length
};

}  // namespace elmm
