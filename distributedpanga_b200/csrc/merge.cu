// FastGA's self adaptamer seed merge on the GPU: each k-mer table entry's
// seeds found by one thread from a tile of entries staged in shared memory.
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

// A tile of MERGE_TILE entries per CTA, MERGE_ITEMS consecutive entries per
// thread (so a thread's seeds are consecutive in the output), with the LCP
// bytes, contig|strand fields and positions of the tile and of `halo`
// (FREQ + 1) entries on either side staged in shared memory: an entry's run
// lies within FREQ - 1 entries of it, so every read of the scan is there.
template <bool WRITE>
__global__ void __launch_bounds__(MERGE_THREADS)
k_merge(const Rec *__restrict__ rec, const uint8_t *__restrict__ lcp, int64_t n, int freq, int halo,
        uint32_t *__restrict__ blk_n, uint32_t *__restrict__ blk_c, Seed *__restrict__ nseed,
        Seed *__restrict__ cseed, int ctgb) {
  extern __shared__ __align__(16) unsigned char msm[];
  __shared__ uint32_t sm[33];
  const int span = MERGE_TILE + 2 * halo;
  uint32_t *spos = reinterpret_cast<uint32_t *>(msm);
  uint16_t *scs = reinterpret_cast<uint16_t *>(spos + span);
  uint8_t *slcp = reinterpret_cast<uint8_t *>(scs + span);
  const int64_t t0 = (int64_t)blockIdx.x * MERGE_TILE, g0 = t0 - halo;  // entry of slot 0
  for (int q = threadIdx.x; q < span; q += MERGE_THREADS) {
    const int64_t g = g0 + q;
    const bool in = g >= 0 && g < n;
    const uint64_t lo = in ? rec[g].lo : 0ull;
    if (WRITE) spos[q] = (uint32_t)lo;
    scs[q] = (uint16_t)(lo >> 32);
    slcp[q] = in ? lcp[g] : 0;
  }
  __syncthreads();
  const uint32_t sbit = 1u << (8 * ctgb - 1);
  uint32_t cn = 0, cc = 0;
  int rs[MERGE_ITEMS], rt[MERGE_ITEMS], rp[MERGE_ITEMS];
#pragma unroll
  for (int e = 0; e < MERGE_ITEMS; e++) {
    rs[e] = rt[e] = 0;
    rp[e] = -1;
    const int64_t i = t0 + (int64_t)threadIdx.x * MERGE_ITEMS + e;
    if (i >= n) continue;
    const int x = (int)(i - g0);  // slot of i
    const int li = slcp[x], ln = i + 1 < n ? slcp[x + 1] : 0;
    const int plen = li > ln ? li : ln;
    if (plen < 12) continue;
    // run start: the last r <= i with lcp[r] < plen, or the table's first entry
    int64_t s = i;
    bool cut = false;
    while (s > 0 && slcp[s - g0] >= plen) {
      s--;
      if (i + 1 - s >= freq) {
        cut = true;
        break;
      }
    }
    if (cut) continue;
    // run end: the first t > i with lcp[t] < plen
    int64_t t = i + 1;
    while (t < n && slcp[t - g0] >= plen) {
      t++;
      if (t - s >= freq) {
        cut = true;
        break;
      }
    }
    if (cut || t - s >= freq) continue;
    rs[e] = (int)(s - g0);
    rt[e] = (int)(t - g0);
    rp[e] = plen;
    const uint32_t si = scs[x] & sbit;
    for (int y = rs[e]; y < rt[e]; y++) {
      if (y == x) continue;
      if ((scs[y] & sbit) == si) cn++;
      else cc++;
    }
  }
  uint32_t tn, tc;
  const uint32_t on = block_exclusive_scan<uint32_t>(cn, sm, &tn);
  const uint32_t oc = block_exclusive_scan<uint32_t>(cc, sm, &tc);
  if (!WRITE) {
    if (threadIdx.x == 0) {
      blk_n[blockIdx.x] = tn;
      blk_c[blockIdx.x] = tc;
    }
    return;
  }
  uint64_t wn = (uint64_t)blk_n[blockIdx.x] + on, wc = (uint64_t)blk_c[blockIdx.x] + oc;
#pragma unroll
  for (int e = 0; e < MERGE_ITEMS; e++) {
    if (rp[e] < 0) continue;
    const int x = threadIdx.x * MERGE_ITEMS + e + halo;
    const uint32_t csi = scs[x];
    const uint64_t ipos = spos[x], icont = csi & (sbit - 1u);
    for (int y = rs[e]; y < rt[e]; y++) {
      if (y == x) continue;
      const uint32_t csj = scs[y];
      Seed sd;
      sd.a = ipos | ((uint64_t)spos[y] << 32);
      sd.b = icont | ((uint64_t)csj << 16) | ((uint64_t)rp[e] << 32);
      if ((csi & sbit) == (csj & sbit)) nseed[wn++] = sd;
      else cseed[wc++] = sd;
    }
  }
}

size_t merge_smem(int freq) { return (size_t)(MERGE_TILE + 2 * (freq + 1)) * 7; }

cudaError_t launch_merge(bool write, int nb, cudaStream_t st, const Rec *rec, const uint8_t *lcp, int64_t n, int freq,
                         uint32_t *blk_n, uint32_t *blk_c, Seed *nseed, Seed *cseed, int ctgb) {
  if (nb <= 0) return cudaSuccess;
  const size_t smem = merge_smem(freq);
  const int halo = freq + 1;
  if (write) {
    cudaError_t e = cudaFuncSetAttribute(k_merge<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_merge<true><<<nb, MERGE_THREADS, smem, st>>>(rec, lcp, n, freq, halo, blk_n, blk_c, nseed, cseed, ctgb);
  } else {
    cudaError_t e = cudaFuncSetAttribute(k_merge<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_merge<false><<<nb, MERGE_THREADS, smem, st>>>(rec, lcp, n, freq, halo, blk_n, blk_c, nseed, cseed, ctgb);
  }
  return cudaGetLastError();
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
