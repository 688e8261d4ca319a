// af_arena.cpp -- the arena planner (see af_arena.h) and its C test/planning
// entry points (af_arena_* in include/adaptflood.h).
#include "af_arena.h"

#include <new>

#include "adaptflood.h"

namespace af {

void Arena::reset(uint64_t bytes) {
  size_ = bytes / kAlign * kAlign;
  used_ = 0;
  free_by_off_.clear();
  free_by_len_.clear();
  used_blocks_.clear();
  if (size_ > 0) insert_free(0, size_);
}

void Arena::insert_free(uint64_t off, uint64_t len) {
  free_by_off_[off] = len;
  free_by_len_.insert({len, off});
}

void Arena::erase_free(uint64_t off, uint64_t len) {
  free_by_off_.erase(off);
  free_by_len_.erase({len, off});
}

bool Arena::alloc(uint64_t bytes, uint64_t* off) {
  if (bytes == 0) bytes = 1;
  if (bytes > size_) return false;
  const uint64_t need = (bytes + kAlign - 1) / kAlign * kAlign;
  // Best fit: the smallest free block that holds `need` (lowest offset on ties).
  auto it = free_by_len_.lower_bound({need, 0});
  if (it == free_by_len_.end()) return false;
  const uint64_t len = it->first, at = it->second;
  erase_free(at, len);
  if (len > need) insert_free(at + need, len - need);
  used_blocks_[at] = need;
  used_ += need;
  *off = at;
  return true;
}

bool Arena::release(uint64_t off) {
  auto u = used_blocks_.find(off);
  if (u == used_blocks_.end()) return false;
  uint64_t at = off, len = u->second;
  used_blocks_.erase(u);
  used_ -= len;
  // Coalesce with the free neighbours on either side.
  auto nx = free_by_off_.lower_bound(at);
  if (nx != free_by_off_.end() && nx->first == at + len) {
    const uint64_t nlen = nx->second;
    erase_free(nx->first, nlen);
    len += nlen;
  }
  auto pv = free_by_off_.lower_bound(at);
  if (pv != free_by_off_.begin()) {
    --pv;
    if (pv->first + pv->second == at) {
      const uint64_t poff = pv->first, plen = pv->second;
      erase_free(poff, plen);
      at = poff;
      len += plen;
    }
  }
  insert_free(at, len);
  return true;
}

uint64_t Arena::largest_free() const {
  return free_by_len_.empty() ? 0 : free_by_len_.rbegin()->first;
}

}  // namespace af

struct af_arena {
  af::Arena a;
};

extern "C" {

int af_arena_create(uint64_t bytes, af_arena** out) {
  if (!out) return AF_EINVAL;
  af_arena* h = new (std::nothrow) af_arena;
  if (!h) return AF_ENOMEM;
  h->a.reset(bytes);
  *out = h;
  return AF_OK;
}

int af_arena_destroy(af_arena* h) {
  if (!h) return AF_EINVAL;
  delete h;
  return AF_OK;
}

int af_arena_alloc(af_arena* h, uint64_t bytes, uint64_t* off) {
  if (!h || !off) return AF_EINVAL;
  return h->a.alloc(bytes, off) ? AF_OK : AF_ENOMEM;
}

int af_arena_free(af_arena* h, uint64_t off) {
  if (!h) return AF_EINVAL;
  return h->a.release(off) ? AF_OK : AF_EINVAL;
}

int af_arena_stats(const af_arena* h, uint64_t* used, uint64_t* largest_free, int* blocks) {
  if (!h) return AF_EINVAL;
  if (used) *used = h->a.used();
  if (largest_free) *largest_free = h->a.largest_free();
  if (blocks) *blocks = h->a.blocks();
  return AF_OK;
}

}  // extern "C"
