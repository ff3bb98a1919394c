// arena.h -- first-fit sub-allocator over one device memory range.
//
// The serving loop reserves its whole HBM budget once and carves every job's
// buffers out of it: admission is then a question of whether a job's
// footprint fits, and no cudaMalloc / cudaFree (whose implicit device
// synchronisation would stall the jobs already running) happens while jobs
// are in flight.  Blocks are aligned to 512 bytes; freed blocks coalesce with
// their neighbours.  The arena only does address arithmetic, so it is tested
// on any base value without a GPU.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <map>
#include <mutex>

class Arena {
 public:
  static constexpr size_t kAlign = 512;

  Arena(uintptr_t base, size_t bytes) : base_(base), size_(bytes / kAlign * kAlign) {
    if (size_) free_[0] = size_;
  }

  // Returns the address of a block of at least `bytes`, or 0 when no free
  // range is large enough.
  uintptr_t alloc(size_t bytes) {
    std::lock_guard<std::mutex> g(mu_);
    const size_t need = round(bytes ? bytes : 1);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < need) continue;
      const size_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > need) free_[off + need] = len - need;
      used_[off] = need;
      in_use_ += need;
      return base_ + off;
    }
    return 0;
  }

  // Returns false if `p` is not a live block of this arena.
  bool release(uintptr_t p) {
    std::lock_guard<std::mutex> g(mu_);
    if (p < base_) return false;
    auto u = used_.find(p - base_);
    if (u == used_.end()) return false;
    size_t off = u->first, len = u->second;
    used_.erase(u);
    in_use_ -= len;
    auto nx = free_.lower_bound(off);
    if (nx != free_.end() && nx->first == off + len) {   // merge the next range
      len += nx->second;
      nx = free_.erase(nx);
    }
    if (nx != free_.begin()) {                            // merge the previous range
      auto pv = std::prev(nx);
      if (pv->first + pv->second == off) {
        pv->second += len;
        return true;
      }
    }
    free_[off] = len;
    return true;
  }

  size_t capacity() const { return size_; }
  size_t in_use() const {
    std::lock_guard<std::mutex> g(mu_);
    return in_use_;
  }
  size_t largest_free() const {
    std::lock_guard<std::mutex> g(mu_);
    size_t m = 0;
    for (const auto &f : free_) m = f.second > m ? f.second : m;
    return m;
  }
  int free_ranges() const {
    std::lock_guard<std::mutex> g(mu_);
    return (int)free_.size();
  }
  static size_t round(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

 private:
  uintptr_t base_;
  size_t size_;
  size_t in_use_ = 0;
  std::map<size_t, size_t> free_;   // offset -> length
  std::map<size_t, size_t> used_;   // offset -> length
  mutable std::mutex mu_;
};
