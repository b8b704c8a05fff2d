// Device-wide exclusive prefix sum (reduce -> scan of block totals -> scan),
// used for bucket starts, per-tile record offsets and seed offsets.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pga {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *smem, T *total) {
  // smem: SCAN_THREADS/32 + 1 elements
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    T w = lane < nw ? smem[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) smem[lane] = w;
    if (lane == nw - 1) smem[32] = w;
  }
  __syncthreads();
  T pre = (warp > 0 ? smem[warp - 1] : T(0)) + x - v;
  if (total) *total = smem[32];
  __syncthreads();
  return pre;
}

template <typename T>
__global__ void k_scan_reduce(const T *__restrict__ in, int64_t n, T *__restrict__ block_sums) {
  __shared__ T sm[33];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  T s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    int64_t i = base + (int64_t)k * SCAN_THREADS + threadIdx.x;
    if (i < n) s += in[i];
  }
  T tot;
  block_exclusive_scan<T>(s, sm, &tot);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

template <typename T>
__global__ void k_scan_blocks(T *__restrict__ block_sums, int64_t nb, T *__restrict__ total) {
  __shared__ T sm[33];
  T carry = 0;
  for (int64_t b0 = 0; b0 < nb; b0 += SCAN_THREADS) {
    int64_t i = b0 + threadIdx.x;
    T v = i < nb ? block_sums[i] : T(0);
    T tot;
    T p = block_exclusive_scan<T>(v, sm, &tot);
    if (i < nb) block_sums[i] = carry + p;
    carry += tot;
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

template <typename T>
__global__ void k_scan_apply(const T *__restrict__ in, int64_t n, const T *__restrict__ block_sums,
                             T *__restrict__ out) {
  __shared__ T sm[33];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
  T v[SCAN_ITEMS];
  T s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    int64_t i = base + k;
    v[k] = i < n ? in[i] : T(0);
    s += v[k];
  }
  T p = block_exclusive_scan<T>(s, sm, (T *)nullptr) + block_sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    int64_t i = base + k;
    if (i < n) out[i] = p;
    p += v[k];
  }
}

// out[i] = sum(in[0..i)), *total = sum(in) (device pointer, may be null).
// `tmp` needs scan_tmp_elems(n) elements.  in and out may alias.
inline int64_t scan_tmp_elems(int64_t n) { return (n + SCAN_TILE - 1) / SCAN_TILE + 1; }

template <typename T>
cudaError_t exclusive_scan(const T *in, T *out, int64_t n, T *tmp, T *total, cudaStream_t st) {
  int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (nb == 0) {
    if (total) return cudaMemsetAsync(total, 0, sizeof(T), st);
    return cudaSuccess;
  }
  k_scan_reduce<T><<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, n, tmp);
  k_scan_blocks<T><<<1, SCAN_THREADS, 0, st>>>(tmp, nb, total);
  k_scan_apply<T><<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, n, tmp, out);
  return cudaGetLastError();
}

}  // namespace pga
