// Index-build kernels (index.cu) and their launch constants.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

namespace pga {

enum { EXT_COUNT = 0, EXT_WRITE = 1, EXT_HIST = 2, EXT_DIGIT = 3 };

// Two-level bucketing of the extracted records.  EXT_HIST counts records per
// digit (the top `dbits` bits of the 24-bit prefix: 18, wider only when the
// digits would average more than DS_CAP_MID records -- at 2 x 1 Gbp, 21-bit
// digits measured slower than 18-bit ones: their 2^21 write fronts do not fit
// in L2 and 2^21 short CTAs cost more than the overflow classes save);
// EXT_DIGIT writes each record into
// its digit's region -- where its prefix buckets lie in the sorted index --
// through one cursor per digit (the write fronts stay in L2, which merges the
// 16-byte writes into whole lines); k_digit_sort then sorts every digit's
// region in shared memory and writes the prefix table.  Kernels take the
// digit as dshift = 24 - dbits (the prefix bits below the digit).
constexpr int MIN_DIGIT_BITS = 18;
constexpr int MAX_DIGIT_BITS = 22;
constexpr int MAX_DIGIT_PREFIXES = 1 << (24 - MIN_DIGIT_BITS);  // 24-bit prefixes per digit, at most

// Digit bits for an index of about `records` records.
inline int digit_bits_for(int64_t records) {
  int b = MIN_DIGIT_BITS;
  while (b < MAX_DIGIT_BITS && (records >> b) > 8192) b++;
  return b;
}
constexpr int DS_THREADS = 256;
constexpr int DS_CAP = 2048;                     // records a k_digit_sort CTA sorts (36 KB of shared memory)
constexpr int DS_MID_THREADS = 1024;
constexpr int DS_CAP_MID = 8192;                 // the same for the digits above DS_CAP (144 KB)
constexpr int BD_THREADS = 1024;                 // k_big_digit

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
                    uint32_t *counts, const uint64_t *offsets, Rec *out, uint32_t *hist, uint32_t *cursor,
                    int dshift = 0);
__global__ void k_prefix_hist(const Rec *rec, int64_t n, uint32_t *hist);
__global__ void k_prefix_scatter(const Rec *in, int64_t n, uint32_t *cursor, Rec *out);
// Sorts the region of digit d (list[blockIdx.x], or blockIdx.x when list is
// null) in place when it holds at most cap (DS_CAP or DS_CAP_MID) records and writes start[] for its 2^dshift prefixes; a larger digit
// is appended to qnext (count *qnext_count).
cudaError_t launch_digit_sort(int cap, int grid, int threads, cudaStream_t st, Rec *rec, const uint32_t *dstart,
                              uint32_t *start, const uint32_t *list, uint32_t *qnext, uint32_t *qnext_count,
                              int dshift);
// One CTA per digit of `list` (scratch for list[i] at tmp_all + toff[i]):
// start[] for its prefixes, records grouped by prefix, buckets of more than
// one record queued for k_bucket_medium / k_bucket_big_step.
__global__ void k_big_digit(Rec *rec, const uint32_t *dstart, uint32_t *start, const uint32_t *list,
                            const int64_t *toff, Rec *tmp_all, uint32_t *qmed, uint32_t *qbig, uint32_t *qcount,
                            int dshift);
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
// The union of sorted indices a (prefix table sa, contig|strand width actgb
// <= ctgb) and b (sb, ctgb) with no record in common, written to out in order.
__global__ void k_union_rank(const Rec *a, const uint32_t *sa, int64_t na, int actgb, const Rec *b,
                             const uint32_t *sb, int64_t nb, int ctgb, Rec *out);
// start[p] += other[p] for p in [0, NPREFIX].
__global__ void k_add_prefix_tables(uint32_t *start, const uint32_t *other);

}  // namespace pga
