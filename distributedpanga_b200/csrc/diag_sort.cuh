// Diagonal sort of one seed unit for the resident pipeline (diag_sort.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"
#include "seeds.cuh"

namespace pga {

constexpr int DSP_THREADS = 256;
constexpr int DSP_ITEMS = 16;
constexpr int DSP_TILE = DSP_THREADS * DSP_ITEMS;

// Bytes of the small scratch a sort needs (histograms, digit starts, tile
// counters, key bit summaries, error flag).
constexpr size_t DIAG_SORT_SMALL = 96 * 1024;

// Bytes of the look-back words of one pass over n keys.
inline size_t diag_sort_look_bytes(int64_t n) {
  return sizeof(unsigned long long) * 256 * (size_t)((n + DSP_TILE - 1) / DSP_TILE) + 64;
}

struct DiagSortResult {
  bool in_a;       // the sorted 128-bit keys are in buffer a (else b)
  int passes;      // digit passes run
  int launches;    // kernels launched
  int bad;         // 1: a pass gave up waiting for a tile before it (no result)
};

// Sorts the diagonal-sort keys of seeds sd[0..n) (layout L): a holds the
// seeds on entry and is overwritten; a and b each hold at least 16 n + 16
// bytes.  The sorted keys (U128, ascending) end in a or b.  look:
// diag_sort_look_bytes(n); small: DIAG_SORT_SMALL bytes.  Synchronizes the
// stream twice (the key bits, and the error flag at the end).
cudaError_t diag_sort_seeds(void *a, void *b, int64_t n, const SeedKeyLayout &L, unsigned long long *look,
                            void *small, cudaStream_t st, DiagSortResult *res);

}  // namespace pga
