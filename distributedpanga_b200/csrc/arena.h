// Device memory of one context: slabs taken from the driver once, carved
// into buffers, freed ranges kept and coalesced for the next request.
//
// A pipeline pass frees and requests the same buffer sizes in the same order
// every time (the index, then the seeds, then the sort keys; the alignment's
// buffers in the space the index and seeds leave), so after the first pass
// every request is met from ranges the arena already holds and the pass makes
// no cudaMalloc / cudaFree calls.  On a 2 x 1 Gbp genome pair those calls
// took about 0.9 s of a 4.9 s pass (page mapping of ~100 GB a pass).
//
// Requests below SMALL_LIMIT share SMALL_SLAB-sized slabs; larger ones take
// the best-fitting free range of a large slab, else a new slab of their own
// size.  When the driver has no room, slabs with nothing live in them go
// back to it and the request is retried; a caller that can free buffers of
// its own (the context's alignment buffers) does so and asks again.
//
// Host-only: the driver's allocate / free are function pointers, so the
// placement logic is tested on the CPU with a fake device.
#pragma once
#include <cstddef>
#include <cstdint>
#include <map>
#include <vector>

namespace pga {

class Arena {
 public:
  // 0 on success; *p is then at least 256-byte aligned
  using MallocFn = int (*)(void *user, void **p, size_t bytes);
  using FreeFn = void (*)(void *user, void *p);

  static constexpr size_t ALIGN = 256;
  static constexpr size_t SMALL_LIMIT = (size_t)32 << 20;
  static constexpr size_t SMALL_SLAB = (size_t)256 << 20;
  static constexpr size_t LARGE_GRAIN = (size_t)2 << 20;

  Arena(MallocFn m, FreeFn f, void *user) : m_(m), f_(f), user_(user) {}
  Arena(const Arena &) = delete;
  Arena &operator=(const Arena &) = delete;
  ~Arena() { clear(); }

  // A buffer of at least `bytes`: a held range if one fits, else a new slab.
  // nullptr when neither works after empty slabs went back to the driver.
  void *alloc(size_t bytes) {
    const size_t need = round_up(bytes ? bytes : 1, ALIGN);
    if (void *p = fit(need)) return p;
    if (grow(need)) return fit(need);
    if (trim() && grow(need)) return fit(need);
    return nullptr;
  }

  // A held range of at least `bytes`, or nullptr (no driver call).
  void *fit(size_t bytes) {
    const size_t need = round_up(bytes ? bytes : 1, ALIGN);
    const bool small = need < SMALL_LIMIT;
    int bs = -1;
    size_t boff = 0, blen = 0;
    for (int s = 0; s < (int)slabs_.size(); s++) {
      const Slab &S = slabs_[s];
      if (S.small != small) continue;
      for (const auto &r : S.fr)
        if (r.second >= need && (bs < 0 || r.second < blen)) {
          bs = s;
          boff = r.first;
          blen = r.second;
        }
    }
    if (bs < 0) return nullptr;
    Slab &S = slabs_[bs];
    S.fr.erase(boff);
    if (blen > need) S.fr[boff + need] = blen - need;
    S.live++;
    char *p = S.base + boff;
    live_[p] = {bs, need};
    free_bytes_ -= need;
    return p;
  }

  // Returns a buffer from alloc / fit to its slab.  False if p is not one.
  bool release(void *vp) {
    if (!vp) return true;
    auto it = live_.find((char *)vp);
    if (it == live_.end()) return false;
    const int s = it->second.first;
    const size_t len = it->second.second;
    live_.erase(it);
    Slab &S = slabs_[s];
    size_t off = (size_t)((char *)vp - S.base), n = len;
    auto nx = S.fr.lower_bound(off);
    if (nx != S.fr.end() && nx->first == off + n) {
      n += nx->second;
      nx = S.fr.erase(nx);
    }
    if (nx != S.fr.begin()) {
      auto pv = std::prev(nx);
      if (pv->first + pv->second == off) {
        off = pv->first;
        n += pv->second;
        S.fr.erase(pv);
      }
    }
    S.fr[off] = n;
    S.live--;
    free_bytes_ += len;
    return true;
  }

  // Slabs with nothing live go back to the driver; returns the bytes freed.
  size_t trim() {
    size_t got = 0;
    for (int s = 0; s < (int)slabs_.size(); s++) {
      Slab &S = slabs_[s];
      if (!S.base || S.live) continue;
      f_(user_, S.base);
      driver_calls_++;
      got += S.size;
      held_ -= S.size;
      free_bytes_ -= S.size;
      S = Slab{};
    }
    return got;
  }

  // Frees every slab (the owner frees no buffer after this).
  void clear() {
    for (Slab &S : slabs_)
      if (S.base) {
        f_(user_, S.base);
        driver_calls_++;
      }
    slabs_.clear();
    live_.clear();
    held_ = free_bytes_ = 0;
  }

  size_t held_bytes() const { return held_; }        // in slabs
  size_t free_bytes() const { return free_bytes_; }  // in slabs, not live
  size_t largest_free() const {
    size_t m = 0;
    for (const Slab &S : slabs_)
      for (const auto &r : S.fr) m = r.second > m ? r.second : m;
    return m;
  }
  int slabs() const {
    int n = 0;
    for (const Slab &S : slabs_) n += S.base != nullptr;
    return n;
  }
  int64_t driver_calls() const { return driver_calls_; }

 private:
  struct Slab {
    char *base = nullptr;
    size_t size = 0;
    bool small = false;
    int live = 0;
    std::map<size_t, size_t> fr;  // free ranges: offset -> length
  };

  static size_t round_up(size_t v, size_t g) { return (v + g - 1) / g * g; }

  bool grow(size_t need) {
    const bool small = need < SMALL_LIMIT;
    const size_t size = small ? SMALL_SLAB : round_up(need, LARGE_GRAIN);
    void *p = nullptr;
    driver_calls_++;
    if (m_(user_, &p, size) != 0 || !p) return false;
    Slab S;
    S.base = (char *)p;
    S.size = size;
    S.small = small;
    S.fr[0] = size;
    int slot = -1;
    for (int s = 0; s < (int)slabs_.size(); s++)
      if (!slabs_[s].base) {
        slot = s;
        break;
      }
    if (slot < 0) {
      slabs_.push_back(S);
    } else {
      slabs_[slot] = S;
    }
    held_ += size;
    free_bytes_ += size;
    return true;
  }

  MallocFn m_;
  FreeFn f_;
  void *user_;
  std::vector<Slab> slabs_;
  std::map<char *, std::pair<int, size_t>> live_;  // buffer -> (slab, length)
  size_t held_ = 0, free_bytes_ = 0;
  int64_t driver_calls_ = 0;
};

}  // namespace pga
