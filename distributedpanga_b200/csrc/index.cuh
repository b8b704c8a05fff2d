// Index-build kernels (index.cu) and their launch constants.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

namespace pga {

enum { EXT_COUNT = 0, EXT_WRITE = 1, EXT_HIST = 2, EXT_SCATTER = 3 };

constexpr int EXT_THREADS = 256;                   // threads per extraction CTA
constexpr int EXT_PER = 32;                        // syncmer offsets per thread
constexpr int EXT_TILE = EXT_THREADS * EXT_PER;    // offsets per CTA (multiple of 4)
constexpr int EXT_LEFT = 32;                       // bases staged before the tile (>= 28, multiple of 4)
constexpr int EXT_SPAN = EXT_TILE + 80;            // staged bases (>= EXT_LEFT + EXT_TILE + 40 + 4)

constexpr int BK_RANK_MAX = 256;  // bucket sizes ranked in place by k_bucket_rank
constexpr int BK_MEDIUM = 2048;   // bucket sizes sorted by one CTA in shared memory
constexpr int BK_THREADS = 256;
constexpr int BK_CAP = 4096;      // records a k_bucket_rank CTA stages (64 KB of shared memory)
constexpr int OUT_THREADS = 256;  // records per CTA pass of the byte-format writers

// Launches the extraction kernel in one of the EXT_* modes (one CTA per tile).
void launch_extract(int mode, int ntiles, cudaStream_t st, const uint8_t *bps, const int64_t *clen,
                    const int64_t *boff, const int32_t *tile_ctg, const int64_t *tile_j0, int ctgb,
                    uint32_t *counts, const uint64_t *offsets, Rec *out, uint32_t *hist, uint32_t *cursor);
__global__ void k_prefix_hist(const Rec *rec, int64_t n, uint32_t *hist);
__global__ void k_prefix_scatter(const Rec *in, int64_t n, uint32_t *cursor, Rec *out);
__global__ void k_bucket_rank(Rec *rec, const uint32_t *start, int bpc, int cap, uint32_t *qmed,
                              uint32_t *qbig, uint32_t *qcount);
__global__ void k_bucket_medium(Rec *rec, const uint32_t *start, const uint32_t *qmed);
__global__ void k_bucket_big_step(Rec *rec, const uint32_t *start, const uint32_t *qbig, uint32_t k,
                                  uint32_t j);
__global__ void k_lcp(const Rec *rec, int64_t n, uint8_t *lcp);
__global__ void k_entries(const Rec *rec, const uint8_t *lcp, int64_t n, int posb, int ctgb, uint8_t *ent);
__global__ void k_records_out(const Rec *rec, const uint8_t *lcp, int64_t n, int posb, int ctgb,
                              uint8_t *out);
__global__ void k_records_in(const uint8_t *in, int64_t n, int posb, int ctgb, Rec *rec, uint8_t *lcp);
__global__ void k_prefix_table(const uint32_t *start, int64_t *cum, uint32_t *maxrun);

}  // namespace pga
