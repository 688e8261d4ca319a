// af_arena.h -- host-side planner of one device memory arena.
//
// The batch engine takes one large device allocation when it is created and
// places every admitted scenario's fields and tables inside it, so admitting
// and retiring scenarios never calls cudaMalloc or cudaFree (cudaFree waits
// for the whole device, which would stall the scenarios still running).  The
// planner only does offset arithmetic on the host: best-fit placement of
// 256-byte-aligned blocks, coalescing of neighbouring free blocks on release.
#pragma once

#include <cstdint>
#include <map>
#include <set>
#include <utility>

namespace af {

class Arena {
 public:
  static constexpr uint64_t kAlign = 256;

  explicit Arena(uint64_t bytes = 0) { reset(bytes); }

  void reset(uint64_t bytes);
  // Places `bytes` (rounded up to kAlign); false when no free block is large
  // enough (nothing changes then).
  bool alloc(uint64_t bytes, uint64_t* off);
  // Releases a block returned by alloc; false for an unknown offset.
  bool release(uint64_t off);

  uint64_t size() const { return size_; }
  uint64_t used() const { return used_; }
  uint64_t largest_free() const;
  int blocks() const { return (int)used_blocks_.size(); }
  int free_blocks() const { return (int)free_by_off_.size(); }

 private:
  void insert_free(uint64_t off, uint64_t len);
  void erase_free(uint64_t off, uint64_t len);

  uint64_t size_ = 0, used_ = 0;
  std::map<uint64_t, uint64_t> free_by_off_;         // offset -> length
  std::set<std::pair<uint64_t, uint64_t>> free_by_len_;  // (length, offset)
  std::map<uint64_t, uint64_t> used_blocks_;         // offset -> length
};

}  // namespace af
