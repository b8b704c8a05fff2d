// Seed reimport + diagonal sort kernels (seeds.cu).
#pragma once
#include <cstdint>
#include "common.cuh"

namespace pga {

// Bit layout of a seed's diagonal-sort key, least significant field first:
// lcp (6 bits), diag & 63 (6), anti, band, jcont, icont.
struct SeedKeyLayout {
  int comp;          // 0: N seeds (same strand), 1: C seeds
  int64_t amxpos, bmxpos, maxdag;
  uint64_t dmask;    // 256^DBYTE - 1: anti and band are stored in DBYTE bytes
  uint64_t jmask;    // contig bits of a contig|strand field
  int dbyte, ctgb;
  int off_dlow, off_anti, off_band, off_j, off_i, w_i, total_bits;
};

__device__ __forceinline__ uint64_t key_bits(const U128 &k, int off, int w) {
  uint64_t v;
  if (off < 64) {
    v = k.lo >> off;
    if (off > 0) v |= k.hi << (64 - off);
  } else {
    v = k.hi >> (off - 64);
  }
  return w >= 64 ? v : (v & ((((uint64_t)1) << w) - 1));
}

__global__ void k_seed_keys(const Seed *sd, int64_t n, SeedKeyLayout L, U128 *keys);
__global__ void k_seed_records(const U128 *keys, int64_t n, SeedKeyLayout L, uint8_t *out);
__global__ void k_panel_bounds(const U128 *keys, int64_t n, SeedKeyLayout L, int ncontig, int64_t *off);

}  // namespace pga
