// The table of a resident target's Local_Alignment calls (the served form's
// record): keys of MEMO_KEY words (the call's inputs), values of MEMO_VAL
// words (its path) and the offset of its trace bytes, in open addressing
// with linear probing over a power-of-two number of slots, at most half
// full; word 0 of an empty slot's key is all ones (a key's word 0 holds two
// contig numbers below 2^15 and a flag, never all ones).
//
// Host-only apart from memo_hash, which the device lookup
// (WarpAligner::call) shares, so the construction is tested on the CPU.
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>

#ifdef __CUDACC__
#define PGA_MEMO_HD __host__ __device__
#else
#define PGA_MEMO_HD
#endif

namespace pga {

constexpr int MEMO_KEY = 6, MEMO_VAL = 6;
constexpr uint32_t MEMO_EMPTY = 0xffffffffu;

PGA_MEMO_HD inline uint64_t memo_hash(const uint32_t *k) {
  uint64_t h = 0x243f6a8885a308d3ull;
  for (int i = 0; i < MEMO_KEY; i++) {
    h ^= k[i];
    h *= 0x9e3779b97f4a7c15ull;
    h ^= h >> 29;
  }
  return h;
}

struct MemoTable {
  std::vector<uint32_t> key;
  std::vector<int32_t> val;
  std::vector<int64_t> toff;
  int64_t cap = 0, entries = 0;
};

// The table of n logged calls: key lk[MEMO_KEY * q ..], value lv[MEMO_VAL *
// q ..], trace offset lt[q] (< 0: the trace was not kept, the call is left
// out).  A key logged more than once keeps its first value (the same call
// has the same result).
inline MemoTable memo_table(const uint32_t *lk, const int32_t *lv, const int64_t *lt, int64_t n) {
  MemoTable T;
  T.cap = 16;
  while (T.cap < 2 * n) T.cap <<= 1;
  T.key.assign(MEMO_KEY * (size_t)T.cap, MEMO_EMPTY);
  T.val.assign(MEMO_VAL * (size_t)T.cap, 0);
  T.toff.assign((size_t)T.cap, 0);
  const uint64_t mask = (uint64_t)T.cap - 1;
  for (int64_t q = 0; q < n; q++) {
    if (lt[q] < 0) continue;
    const uint32_t *k = lk + MEMO_KEY * q;
    for (uint64_t s = memo_hash(k) & mask;; s = (s + 1) & mask) {
      uint32_t *slot = &T.key[MEMO_KEY * s];
      if (slot[0] == MEMO_EMPTY) {
        std::copy(k, k + MEMO_KEY, slot);
        std::copy(lv + MEMO_VAL * q, lv + MEMO_VAL * q + MEMO_VAL, &T.val[MEMO_VAL * s]);
        T.toff[s] = lt[q];
        T.entries++;
        break;
      }
      if (std::equal(k, k + MEMO_KEY, slot)) break;
    }
  }
  return T;
}

// The slot holding key k, or -1: the probe WarpAligner::call makes.
inline int64_t memo_find(const MemoTable &T, const uint32_t *k) {
  const uint64_t mask = (uint64_t)T.cap - 1;
  uint64_t s = memo_hash(k) & mask;
  for (uint64_t probe = 0; probe <= mask; probe++, s = (s + 1) & mask) {
    const uint32_t *q = &T.key[MEMO_KEY * s];
    if (q[0] == MEMO_EMPTY) return -1;
    if (std::equal(k, k + MEMO_KEY, q)) return (int64_t)s;
  }
  return -1;
}

}  // namespace pga
