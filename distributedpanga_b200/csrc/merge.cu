// FastGA's self adaptamer seed merge on the GPU, one thread per k-mer table
// entry.
//
// Reference: new_self_merge_thread / self_adaptamer_merge,
// src/fastga_pipeline.c:245-499.  The reference walks each 24-bit prefix
// group with a stack of run starts (vlcp[]) and an end-of-run flag (eorun).
// That walk gives every entry i the same result as this closed form, which
// needs only the LCPs of the FREQ entries on either side:
//
//   plen(i) = max(lcp[i], lcp[i+1])            longest match of i to any entry
//   run(i)  = maximal [s, t) containing i with lcp[r] >= plen(i) for s < r < t
//   i emits one seed (plen, payload(i), payload(j)) for every j in run(i),
//   j != i, iff t - s < FREQ; to the N unit when i and j are on the same
//   strand, else to C.
//
// (A group's first entry has lcp < 12 and the walk's end-of-group marker is
// 11, so runs never cross a group; an entry alone in its group has
// plen <= 11 and no partner.)  Seeds are written in the reference's emission
// order for a given entry order: entry by entry, partners in table order.
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"
#include "merge.cuh"
#include "scan.cuh"

namespace pga {

struct Run {
  int64_t s, t;
  int plen;
  bool emit;
};

__device__ __forceinline__ Run adaptamer_run(const uint8_t *__restrict__ lcp, int64_t n, int64_t i, int freq) {
  Run r;
  int li = lcp[i];
  int ln = (i + 1 < n) ? lcp[i + 1] : 0;
  r.plen = li > ln ? li : ln;
  r.emit = false;
  r.s = r.t = i;
  if (r.plen < 12) return r;
  // run start: the last r <= i with lcp[r] < plen, or the table's first entry
  int64_t s = i;
  while (s > 0 && lcp[s] >= r.plen) {
    s--;
    if (i + 1 - s >= freq) return r;
  }
  // run end: the first t > i with lcp[t] < plen
  int64_t t = i + 1;
  while (t < n && lcp[t] >= r.plen) {
    t++;
    if (t - s >= freq) return r;
  }
  r.s = s;
  r.t = t;
  r.emit = (t - s) < freq;
  return r;
}

template <bool WRITE>
__global__ void __launch_bounds__(MERGE_THREADS)
k_merge(const Rec *__restrict__ rec, const uint8_t *__restrict__ lcp, int64_t n, int freq,
        uint32_t *__restrict__ blk_n, uint32_t *__restrict__ blk_c,
        Seed *__restrict__ nseed, Seed *__restrict__ cseed, int ctgb) {
  __shared__ uint32_t sm[33];
  const int64_t i = (int64_t)blockIdx.x * MERGE_THREADS + threadIdx.x;
  const uint32_t sbit = 1u << (8 * ctgb - 1);
  uint32_t cn = 0, cc = 0;
  Run r;
  r.emit = false;
  uint32_t cs_i = 0;
  if (i < n) {
    r = adaptamer_run(lcp, n, i, freq);
    if (r.emit) {
      cs_i = rec_cs(rec[i]);
      for (int64_t j = r.s; j < r.t; j++) {
        if (j == i) continue;
        uint32_t cs_j = rec_cs(rec[j]);
        if ((cs_i & sbit) == (cs_j & sbit)) cn++;
        else cc++;
      }
    }
  }
  uint32_t tn, tc;
  uint32_t on = block_exclusive_scan<uint32_t>(cn, sm, &tn);
  uint32_t oc = block_exclusive_scan<uint32_t>(cc, sm, &tc);
  if (!WRITE) {
    if (threadIdx.x == 0) {
      blk_n[blockIdx.x] = tn;
      blk_c[blockIdx.x] = tc;
    }
    return;
  }
  if (!r.emit) return;
  uint64_t wn = (uint64_t)blk_n[blockIdx.x] + on;
  uint64_t wc = (uint64_t)blk_c[blockIdx.x] + oc;
  Rec ri = rec[i];
  uint64_t ipos = rec_pos(ri);
  uint64_t icont = cs_i & (sbit - 1u);
  for (int64_t j = r.s; j < r.t; j++) {
    if (j == i) continue;
    Rec rj = rec[j];
    uint32_t cs_j = rec_cs(rj);
    Seed sd;
    sd.a = ipos | ((uint64_t)rec_pos(rj) << 32);
    sd.b = icont | ((uint64_t)cs_j << 16) | ((uint64_t)r.plen << 32);
    if ((cs_i & sbit) == (cs_j & sbit)) nseed[wn++] = sd;
    else cseed[wc++] = sd;
  }
}

void launch_merge(bool write, int nb, cudaStream_t st, const Rec *rec, const uint8_t *lcp, int64_t n, int freq,
                  uint32_t *blk_n, uint32_t *blk_c, Seed *nseed, Seed *cseed, int ctgb) {
  if (nb <= 0) return;
  if (write)
    k_merge<true><<<nb, MERGE_THREADS, 0, st>>>(rec, lcp, n, freq, blk_n, blk_c, nseed, cseed, ctgb);
  else
    k_merge<false><<<nb, MERGE_THREADS, 0, st>>>(rec, lcp, n, freq, blk_n, blk_c, nseed, cseed, ctgb);
}

// Seeds in the reference's byte format (src/fastga_pipeline.c:391-397):
// [plen][A position, A contig (strand cleared)][B position, B contig|strand].
__global__ void k_seeds_out(const Seed *__restrict__ sd, int64_t n, int posb, int ctgb,
                            uint8_t *__restrict__ out) {
  const int sb = 1 + 2 * (posb + ctgb);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    Seed s = sd[i];
    uint8_t *d = out + i * sb;
    uint64_t ip = s.a & 0xffffffffu, jp = s.a >> 32;
    uint64_t ic = s.b & 0xffffu, jc = (s.b >> 16) & 0xffffu;
    d[0] = (uint8_t)(s.b >> 32);
    int o = 1;
    for (int b = 0; b < posb; b++) d[o++] = (uint8_t)(ip >> (8 * b));
    for (int b = 0; b < ctgb; b++) d[o++] = (uint8_t)(ic >> (8 * b));
    for (int b = 0; b < posb; b++) d[o++] = (uint8_t)(jp >> (8 * b));
    for (int b = 0; b < ctgb; b++) d[o++] = (uint8_t)(jc >> (8 * b));
  }
}

// Seeds in the reference byte format -> Seed.
__global__ void k_seeds_in(const uint8_t *__restrict__ in, int64_t n, int posb, int ctgb,
                           Seed *__restrict__ sd) {
  const int sb = 1 + 2 * (posb + ctgb);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t *d = in + i * sb;
    uint64_t ip = 0, jp = 0, ic = 0, jc = 0;
    int o = 1;
    for (int b = 0; b < posb; b++) ip |= (uint64_t)d[o++] << (8 * b);
    for (int b = 0; b < ctgb; b++) ic |= (uint64_t)d[o++] << (8 * b);
    for (int b = 0; b < posb; b++) jp |= (uint64_t)d[o++] << (8 * b);
    for (int b = 0; b < ctgb; b++) jc |= (uint64_t)d[o++] << (8 * b);
    Seed s;
    s.a = ip | (jp << 32);
    s.b = ic | (jc << 16) | ((uint64_t)d[0] << 32);
    sd[i] = s;
  }
}

}  // namespace pga
