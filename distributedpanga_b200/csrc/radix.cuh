// Stable LSD radix sort of 128-bit keys (keys only), 8-bit digits, used for
// the diagonal sort of seeds.  Only the digit positions in which the keys
// actually differ are sorted (the caller passes them), so a key packed into
// T significant bits costs ceil(T/8) passes.
//
// One pass = k_radix_hist (256-bin histogram per 4096-key tile) -> exclusive
// scan of the digit-major (digit, tile) counts -> k_radix_scatter, which
// ranks keys in their original order inside each tile (warp __match_any_sync
// ranks + per-warp digit counts) so the pass is stable.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "scan.cuh"

namespace pga {

constexpr int RADIX_THREADS = 256;
constexpr int RADIX_ITEMS = 16;
constexpr int RADIX_TILE = RADIX_THREADS * RADIX_ITEMS;

__device__ __forceinline__ uint32_t u128_digit(const U128 &k, int shift) {
  return (uint32_t)(((shift < 64) ? (k.lo >> shift) : (k.hi >> (shift - 64))) & 0xff);
}

static __global__ void k_radix_hist(const U128 *__restrict__ keys, int64_t n, int shift,
                             uint32_t *__restrict__ hist, int nb) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * RADIX_TILE;
  for (int r = 0; r < RADIX_ITEMS; r++) {
    int64_t i = base + (int64_t)r * RADIX_THREADS + threadIdx.x;
    if (i < n) atomicAdd(&h[u128_digit(keys[i], shift)], 1u);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * nb + blockIdx.x] = h[threadIdx.x];
}

static __global__ void k_radix_scatter(const U128 *__restrict__ in, U128 *__restrict__ out, int64_t n,
                                int shift, const uint32_t *__restrict__ offs, int nb) {
  __shared__ uint32_t run[256];
  __shared__ uint32_t wc[RADIX_THREADS / 32][256];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  run[tid] = offs[(int64_t)tid * nb + blockIdx.x];
  const uint32_t lt = (1u << lane) - 1u;
  int64_t base = (int64_t)blockIdx.x * RADIX_TILE;
  for (int r = 0; r < RADIX_ITEMS; r++) {
#pragma unroll
    for (int w = 0; w < RADIX_THREADS / 32; w++) wc[w][tid] = 0;
    __syncthreads();
    int64_t i = base + (int64_t)r * RADIX_THREADS + tid;
    bool valid = i < n;
    U128 k;
    uint32_t d = 256 + lane;  // distinct dummy digits for invalid lanes
    if (valid) {
      k = in[i];
      d = u128_digit(k, shift);
    }
    uint32_t m = __match_any_sync(0xffffffffu, d);
    uint32_t rank = __popc(m & lt);
    if (valid && rank == 0) wc[warp][d] = __popc(m);
    __syncthreads();
    {
      uint32_t s = run[tid];
#pragma unroll
      for (int w = 0; w < RADIX_THREADS / 32; w++) {
        uint32_t c = wc[w][tid];
        wc[w][tid] = s;
        s += c;
      }
      run[tid] = s;
    }
    __syncthreads();
    if (valid) out[wc[warp][d] + rank] = k;
    __syncthreads();
  }
}

// Bits in which any key differs from key 0: OR of (key ^ key0).
static __global__ void k_u128_diffbits(const U128 *__restrict__ keys, int64_t n, unsigned long long *acc) {
  __shared__ unsigned long long slo, shi;
  if (threadIdx.x == 0) { slo = 0; shi = 0; }
  __syncthreads();
  U128 k0 = keys[0];
  uint64_t lo = 0, hi = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    U128 k = keys[i];
    lo |= k.lo ^ k0.lo;
    hi |= k.hi ^ k0.hi;
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo |= __shfl_xor_sync(0xffffffffu, lo, o);
    hi |= __shfl_xor_sync(0xffffffffu, hi, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicOr(&slo, (unsigned long long)lo);
    atomicOr(&shi, (unsigned long long)hi);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicOr(&acc[0], slo);
    atomicOr(&acc[1], shi);
  }
}

// Scratch the sort needs: the second key buffer is separate.
inline int64_t radix_hist_elems(int64_t n) {
  int64_t nb = (n + RADIX_TILE - 1) / RADIX_TILE;
  return 256 * nb;
}

// Sorts keys[0..n) using alt[0..n) as the second buffer.  `passes` lists the
// digit shifts (multiples of 8, ascending).  Returns in *result which of the
// two buffers holds the sorted keys.  hist needs radix_hist_elems(n) and scan
// tmp scan_tmp_elems(radix_hist_elems(n)) uint32 elements.
inline cudaError_t radix_sort_u128(U128 *keys, U128 *alt, int64_t n, const int *passes, int npass,
                                   uint32_t *hist, uint32_t *scan_tmp, U128 **result,
                                   cudaStream_t st) {
  *result = keys;
  if (n <= 1 || npass == 0) return cudaSuccess;
  int nb = (int)((n + RADIX_TILE - 1) / RADIX_TILE);
  U128 *src = keys, *dst = alt;
  for (int p = 0; p < npass; p++) {
    k_radix_hist<<<nb, RADIX_THREADS, 0, st>>>(src, n, passes[p], hist, nb);
    cudaError_t e = exclusive_scan<uint32_t>(hist, hist, (int64_t)256 * nb, scan_tmp,
                                             (uint32_t *)nullptr, st);
    if (e != cudaSuccess) return e;
    k_radix_scatter<<<nb, RADIX_THREADS, 0, st>>>(src, dst, n, passes[p], hist, nb);
    U128 *t = src;
    src = dst;
    dst = t;
  }
  *result = src;
  return cudaGetLastError();
}

}  // namespace pga
