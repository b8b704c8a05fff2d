// Seed reimport and diagonal sort on the GPU.
//
// Reference: reimport_thread (src/fastga_pipeline.c:1391-1450) turns each
// seed into a swide-byte record [lcp][diag & 63][anti][diag >> 6][jcont] in
// the panel of its A contig, and rmsd_sort (lib/RSDsort.c:292-377) sorts
// each panel on the whole record read from its last byte backwards, i.e. by
// (jcont, band, anti, diag & 63, lcp).  Here every seed becomes one 128-bit
// key holding (icont, jcont, band, anti, diag & 63, lcp), most significant
// first, each field in just the bits its range needs, and one stable LSD
// radix sort over the differing digits orders all panels at once.
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"
#include "seeds.cuh"

namespace pga {

__device__ __forceinline__ uint64_t get_bits(const U128 &k, int off, int w) {
  uint64_t v;
  if (off < 64) {
    v = k.lo >> off;
    if (off > 0) v |= k.hi << (64 - off);
  } else {
    v = k.hi >> (off - 64);
  }
  return w >= 64 ? v : (v & ((((uint64_t)1) << w) - 1));
}

__global__ void k_seed_keys(const Seed *__restrict__ sd, int64_t n, SeedKeyLayout L, U128 *__restrict__ keys) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    keys[i] = seed_key(sd[i], L);
}

// Sorted keys -> swide-byte records (src/fastga_pipeline.c:1434-1446).
__global__ void k_seed_records(const U128 *__restrict__ keys, int64_t n, SeedKeyLayout L,
                               uint8_t *__restrict__ out) {
  const int sw = 2 * L.dbyte + L.ctgb + 2;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    U128 k = keys[i];
    uint64_t lcp = get_bits(k, 0, L.off_dlow);
    uint64_t dlow = get_bits(k, L.off_dlow, L.off_anti - L.off_dlow);
    uint64_t anti = get_bits(k, L.off_anti, L.off_band - L.off_anti);
    uint64_t band = get_bits(k, L.off_band, L.off_j - L.off_band);
    uint64_t jc = get_bits(k, L.off_j, L.off_i - L.off_j);
    uint8_t *d = out + i * sw;
    d[0] = (uint8_t)lcp;
    d[1] = (uint8_t)dlow;
    for (int b = 0; b < L.dbyte; b++) d[2 + b] = (uint8_t)(anti >> (8 * b));
    for (int b = 0; b < L.dbyte; b++) d[2 + L.dbyte + b] = (uint8_t)(band >> (8 * b));
    for (int b = 0; b < L.ctgb; b++) d[2 + 2 * L.dbyte + b] = (uint8_t)(jc >> (8 * b));
  }
}

// off[c] = index of the first sorted key whose A contig is >= c, c in
// [0, ncontig]: the panel boundaries (the reference's buck prefix sums).
__global__ void k_panel_bounds(const U128 *__restrict__ keys, int64_t n, SeedKeyLayout L, int ncontig,
                               int64_t *__restrict__ off) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > ncontig) return;
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if ((int64_t)get_bits(keys[mid], L.off_i, L.w_i) < c) lo = mid + 1;
    else hi = mid;
  }
  off[c] = lo;
}

}  // namespace pga
