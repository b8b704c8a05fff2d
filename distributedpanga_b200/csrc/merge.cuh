// Adaptamer merge kernels (merge.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

namespace pga {

constexpr int MERGE_THREADS = 256;
constexpr int MERGE_ITEMS = 4;
constexpr int MERGE_TILE = MERGE_THREADS * MERGE_ITEMS;
// the largest FREQ whose tile (shared memory) the merge launches
constexpr int MERGE_MAX_FREQ = 8192;

// Count (write = false: per-block seed totals) or write pass of the merge:
// nb blocks of MERGE_TILE k-mer table entries, MERGE_ITEMS per thread.
cudaError_t launch_merge(bool write, int nb, cudaStream_t st, const Rec *rec, const uint8_t *lcp, int64_t n, int freq,
                         uint32_t *blk_n, uint32_t *blk_c, Seed *nseed, Seed *cseed, int ctgb);
__global__ void k_seeds_out(const Seed *sd, int64_t n, int posb, int ctgb, uint8_t *out);
__global__ void k_seeds_in(const uint8_t *in, int64_t n, int posb, int ctgb, Seed *sd);

}  // namespace pga
