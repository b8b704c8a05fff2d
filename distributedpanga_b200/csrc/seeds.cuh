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

__device__ __forceinline__ void put_bits(U128 &k, int off, uint64_t v) {
  if (off < 64) {
    k.lo |= v << off;
    if (off > 0) k.hi |= v >> (64 - off);
  } else {
    k.hi |= v << (off - 64);
  }
}

// A seed's diagonal-sort key (reimport_thread's record, src/fastga_pipeline.c:
// 1391-1450, as one integer: icont, jcont, band, anti, diag & 63, lcp from
// the most significant field down).
__device__ __forceinline__ U128 seed_key(const Seed &s, const SeedKeyLayout &L) {
  const int64_t ipost = (int64_t)(s.a & 0xffffffffu), jpost = (int64_t)(s.a >> 32);
  const uint64_t icont = s.b & 0xffffu;
  const uint64_t jcont = ((s.b >> 16) & 0xffffu) & L.jmask;
  const uint64_t lcp = (s.b >> 32) & 0xffu;
  int64_t diag, anti;
  if (L.comp) {
    diag = L.maxdag - (ipost + jpost);
    anti = L.amxpos - (ipost - jpost);
  } else {
    diag = L.bmxpos + (ipost - jpost);
    anti = ipost + jpost;
  }
  const int64_t band = diag >> 6;
  const uint64_t dlow = (uint64_t)(diag - (band << 6)) & 0xffu;
  U128 k = {0, 0};
  put_bits(k, 0, lcp);
  put_bits(k, L.off_dlow, dlow);
  put_bits(k, L.off_anti, (uint64_t)anti & L.dmask);
  put_bits(k, L.off_band, (uint64_t)band & L.dmask);
  put_bits(k, L.off_j, jcont);
  put_bits(k, L.off_i, icont);
  return k;
}

__global__ void k_seed_keys(const Seed *sd, int64_t n, SeedKeyLayout L, U128 *keys);
__global__ void k_seed_records(const U128 *keys, int64_t n, SeedKeyLayout L, uint8_t *out);
__global__ void k_panel_bounds(const U128 *keys, int64_t n, SeedKeyLayout L, int ncontig, int64_t *off);

}  // namespace pga
