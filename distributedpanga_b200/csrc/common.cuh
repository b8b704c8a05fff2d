// Shared definitions for the sm_100a kernels of the alignment path.
//
// Device record layouts (HBM):
//   Rec  (16 B)  one k-mer occurrence of the index.  hi = k-mer bits 79..16
//                (base 0 in bits 63..62), lo = k-mer bits 15..0 << 48 |
//                contig|strand << 32 | position.  Ordering (hi, lo) as
//                unsigned integers sorts by k-mer, then by the reference's
//                payload bytes read as one little-endian integer
//                (contig|strand, then position).
//   Seed (16 B)  one adaptamer seed.  a = A position | B position << 32,
//                b = A contig | B contig|strand << 16 | shared bases << 32.
//
// The reference's byte formats (records, k-mer table entries, seeds, sorted
// seed records) are produced from these only at the C-ABI boundary.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pga {

constexpr int KMER = 40;
constexpr int KBYTES = 10;
constexpr int TMER = 12;
constexpr int NPREFIX = 1 << 24;

struct __align__(16) Rec {
  uint64_t hi;
  uint64_t lo;
};

struct __align__(16) Seed {
  uint64_t a;
  uint64_t b;
};

struct __align__(16) U128 {
  uint64_t lo;
  uint64_t hi;
};

__device__ __forceinline__ bool rec_less(const Rec &x, const Rec &y) {
  return x.hi < y.hi || (x.hi == y.hi && x.lo < y.lo);
}

__device__ __forceinline__ uint32_t rec_prefix(const Rec &r) { return (uint32_t)(r.hi >> 40); }
__device__ __forceinline__ uint32_t rec_pos(const Rec &r) { return (uint32_t)r.lo; }
__device__ __forceinline__ uint32_t rec_cs(const Rec &r) { return (uint32_t)((r.lo >> 32) & 0xffff); }

// Bases in common of two 40-mers, [0, 40].
__device__ __forceinline__ int kmer_lcp(const Rec &a, const Rec &b) {
  uint64_t x = a.hi ^ b.hi;
  if (x) return __clzll(x) >> 1;
  uint32_t y = (uint32_t)((a.lo ^ b.lo) >> 48);
  if (y) return 32 + ((__clz(y) - 16) >> 1);
  return KMER;
}

}  // namespace pga

#define PGA_CUDA_TRY(x)                         \
  do {                                          \
    cudaError_t _e = (x);                       \
    if (_e != cudaSuccess) return _e;           \
  } while (0)
