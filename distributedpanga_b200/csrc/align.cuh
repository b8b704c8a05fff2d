// Alignment-stage launch description and records (align.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "align_core.cuh"
#include "common.cuh"
#include "seeds.cuh"
#include "memo.h"

namespace pga {

constexpr int ALIGN_THREADS = 128;  // 4 warps per CTA, one pair per warp at a time
constexpr int WAVE_INTS = 13;       // per diagonal slot: V,M,HA,HM x2, NA, T x2 (uint64)

// One (anchor, partner) pair of a unit: seeds [lo, hi) of the unit's sorted
// keys.  seg < 0: the whole pair, finished by the same warp.  seg >= 0: band
// range number seg of a pair run in ranges: the band blocks whose first
// stream starts in [slo, shi), both moved forward to the next band start;
// its candidates go to the range store, its PairOut to rout[seg], and
// k_finish_pairs finishes the pair later.
struct PairTask {
  int comp, a, b, self, entry_bepos, seg;
  int64_t lo, hi, slo, shi;
};

// Per task.  For a range task nsurv is its candidate count and rec_off the
// offset of its candidates in the range store.
struct PairOut {
  int calls, exit_bepos, nsurv, err;
  int64_t rec_off;
  long long cycles;     // SM clock cycles the warp spent on the task
  int64_t waves, cells;  // wave steps of its Local_Alignment calls, and their diagonals
};

// A pair run in ranges: its ranges, in order, are range_idx[first ..
// first + nseg).
struct FinishTask {
  int comp, a, b, entry_bepos, first, nseg;
};

// One surviving alignment; trace bytes (uint8 pairs: diffs, b-delta per
// trace interval) at toff in the output byte array.
struct AlnRec {
  int aread, bread, comp, abpos, aepos, bbpos, bepos, diffs, tlen, rank;
  int64_t toff;
};

// A resident target's Local_Alignment results (pga_target_create_reuse).
// A call's result -- the path and its trace points -- is a function of its
// inputs: the two contigs (their bases), the orientation, low, hgh, anti,
// lbord, hbord, and the scoring tables.  The target's own run appends every
// call to a log (capture); a request's calls on two target contigs look
// their inputs up in a table built from it and take the recorded result
// instead of running the wave loop.
struct CallMemo {
  // table of cap slots (a power of two; 0: none), MEMO_KEY words of key per
  // slot (word 0 all ones: empty), MEMO_VAL of value (abpos, aepos, bbpos,
  // bepos, diffs, tlen), and the offset of its trace bytes in trace
  const uint32_t *key;
  const int32_t *val;
  const int64_t *toff;
  const uint8_t *trace;
  int64_t cap;
  int nt;                      // the target's contigs: 0 .. nt-1
  unsigned long long *hits;    // calls answered from the table
  // capture log (lkey null: off): up to lcap calls, lbytes_cap trace bytes
  uint32_t *lkey;
  int32_t *lval;
  int64_t *ltoff;
  uint8_t *ltrace;
  unsigned long long *lnext, *lbytes;
  int64_t lcap, lbytes_cap;
};

struct AlignLaunch {
  const PairTask *tasks;
  int ntasks;
  unsigned *next_task;
  unsigned *smflag;   // k_align_pairs: SM_FLAGS flags, zero at launch (null: off)
  // SM cycles the launch's warps spent in Local_Alignment [0] and in the
  // pairs' finishing step [1], zero at launch
  unsigned long long *prof;
  CallMemo memo;
  int long_waves;     // a wave loop past this many waves flags its SM
  const U128 *keysN, *keysC;
  // per seed of each unit: band start (bit 15), previous band of the pair
  // adjacent (bit 14), capped 2*lcp sum of the band at its start (bits 0-7)
  const uint16_t *infoN, *infoC;
  SeedKeyLayout layN, layC;
  const uint8_t *fwd, *rc;
  const int64_t *soff, *clen;
  const uint64_t *pk;            // packed sequences: contig c at word 4*poff[c]: F, R, RC, CO (pwords[c] each)
  const int64_t *poff, *pwords;
  const int16_t *score, *table;
  int ave_path;
  int64_t amxpos, maxdag;
  int64_t nwarps;
  int *wave;
  int vcap;
  uint16_t *points;
  int64_t point_cap;
  aln::Pebble *cells;
  unsigned long long *cell_next;
  int64_t cell_cap;
  aln::Ovl *ovl;
  int *perm;  // 2 * ovl_cap ints per warp: the order and the merge sort's buffer
  int64_t ovl_cap;
  aln::Ovl *rng_ovl;                 // range store: candidates of range tasks
  unsigned long long *rng_next;
  int64_t rng_cap;
  PairOut *rout;                     // per range number
  const int32_t *lreq;               // k_local_batch: 8 ints per request
  int64_t nlreq;
  unsigned long long *lreq_next;
  int32_t *lpath;                    // 7 ints per request
  int64_t *ltoff;                    // trace offset per request (-1: none)
  uint16_t *ltrace;
  unsigned long long *ltrace_next;
  int64_t ltrace_cap;
  const FinishTask *ftasks;          // k_finish_pairs
  int nftasks;
  const int *range_idx;
  uint8_t *cand_bytes;
  unsigned long long *cand_next;
  int64_t cand_cap;
  PairOut *pout;
  AlnRec *recs;
  unsigned long long *rec_next;
  int64_t rec_cap;
  uint8_t *out_bytes;
  unsigned long long *out_next;
  int64_t out_cap;
  // Pairs planned on the device: task t >= ntasks is pair small[t - ntasks]
  // (bit 63 its unit, the rest its index in that unit's pair list: seeds
  // pstart[u][p] .. pstart[u][p + 1] (or nseeds[u]), contigs pab[u][2p],
  // pab[u][2p + 1]).  Their outcomes are reduced instead of stored:
  // sred = {calls, cycles, max (cycles << 16 | calls), error bits, waves,
  // cells, first failing task}; per FastGA order position of an N pair's
  // anchor, fo_last = the largest fo key (b position + 1 << 32 | exit
  // bepos) of its pairs that called and fo_earlier = the same over partners
  // ordered before the anchor.
  const uint64_t *small;
  int nsmall;
  const int64_t *pstart[2];
  const int32_t *pab[2];
  int64_t npairs[2], nseeds[2];
  const int *fo_pos;
  unsigned long long *sred, *fo_last, *fo_earlier;
  // build of k_align_pairs: 2 (all registers), 3, 4 or 5 resident CTAs per SM
  int min_blocks;
};

// Pair lists on the device: whether the host plans pair p of a unit (a self
// pair, or one of more than rs seeds when rs > 0), the host's list, and the
// other pairs that can make a Local_Alignment call (their seeds' spans reach
// CHAIN_MIN) as `small` codes, largest first (sizes clamped to 65535).
constexpr int SMALL_BINS = 65536;
void launch_pair_hostbound(const int64_t *pstart, const int32_t *pab, int64_t np, int64_t nseeds, int comp, int64_t rs,
                           uint32_t *flag, cudaStream_t st);
void launch_pair_gather(const int64_t *pstart, const int32_t *pab, int64_t np, int64_t nseeds, const uint32_t *flag,
                        const uint32_t *idx, int64_t *out3, cudaStream_t st);
void launch_pair_live(const uint16_t *info, int64_t n, const uint32_t *pflag, const uint32_t *pidx, uint8_t *live,
                      cudaStream_t st);
void launch_small_hist(const int64_t *pstart, const int32_t *pab, int64_t np, int64_t nseeds, int comp, int64_t rs,
                       const uint8_t *live, uint32_t *hist, cudaStream_t st);
void launch_small_scatter(const int64_t *pstart, const int32_t *pab, int64_t np, int64_t nseeds, int comp, int64_t rs,
                          const uint8_t *live, uint32_t *cursor, uint64_t *small, cudaStream_t st);

void launch_align(const AlignLaunch &P, int grid, cudaStream_t st);
void launch_finish(const AlignLaunch &P, int grid, cudaStream_t st);
void launch_local_batch(const AlignLaunch &P, int grid, cudaStream_t st);
void launch_self_bounds(const U128 *keys, SeedKeyLayout L, const int64_t *lohi, int npair, int64_t cd_lo,
                        int64_t cd_hi, int64_t *x12, cudaStream_t st);
void launch_base_counts(const uint8_t *bps, const int64_t *clen, const int64_t *boff, int ncontig,
                        unsigned long long *cnt, cudaStream_t st);
void launch_numeric(const uint8_t *bps, const int64_t *clen, const int64_t *boff, const int64_t *soff, int ncontig,
                    uint8_t *fwd, uint8_t *rc, cudaStream_t st);
void launch_pack(const uint8_t *fwd, const int64_t *soff, const int64_t *clen, const int64_t *poff,
                 const int64_t *pwords, int ncontig, uint64_t *pk, cudaStream_t st);
void launch_band_info(const U128 *keys, int64_t n, SeedKeyLayout L, uint16_t *info, cudaStream_t st);
void launch_pair_flags(const U128 *keys, int64_t n, SeedKeyLayout L, uint32_t *flag, cudaStream_t st);
void launch_pair_starts(const U128 *keys, int64_t n, SeedKeyLayout L, const uint32_t *flag, const uint32_t *idx,
                        int64_t *start, int32_t *ab, cudaStream_t st);
// la_sort order of the surviving alignments on the device: keys, then (after
// the keys are sorted) the records in that order with their trace lengths,
// then the traces moved to the scanned offsets.
void launch_aln_keys(const AlnRec *r, int64_t n, U128 *keys, cudaStream_t st);
void launch_aln_gather(const U128 *keys, int64_t n, const AlnRec *in, AlnRec *out, int64_t *len, cudaStream_t st);
void launch_aln_traces(AlnRec *recs, const int64_t *off, int64_t n, const uint8_t *src, uint8_t *dst,
                       cudaStream_t st);


}  // namespace pga
