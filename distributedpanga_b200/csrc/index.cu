// Index build on the GPU: closed-syncmer extraction from the 2-bit GDB,
// bucketing by the 24-bit k-mer prefix, in-bucket sort, semantic LCPs, the
// k-mer table entries and the 2^24 cumulative prefix table.
//
// Reference path replaced (one process, world size 1):
//   extract_to_records     src/extract.c:85-358, src/pack.c:29-78
//   run_stage2 sort + LCP  src/dsort.c:369-518, src/sort.c:38-115, lib/MSDsort.c:404-507
//   build_kmer_adapter     src/kmer_adapter.c:6-96
//
// The MPI bucket exchange of run_stage2 becomes an in-HBM MSD sort in two
// levels: a histogram of the digits (the first 9 bases, more for very large
// indexes), a scatter of
// every record into its digit's region as it is extracted, then a sort of
// each digit's region in shared memory that also writes the 24-bit prefix
// table (the k-mer table's cumulative prefix index).  Records extracted from
// the host's byte format go through the one-level path: prefix histogram,
// scatter into the prefix buckets, per-bucket finishing sort.
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"
#include "index.cuh"

namespace pga {

// The syncmer hash's 4-mer scramble table (src/tables.c:5-22); part of the
// selection rule's definition, so the values are the reference's.
__constant__ uint8_t c_tmap[256] = {
  0xff,0xd4,0xf5,0xfd,0xe4,0xad,0x21,0xa5,0xed,0x64,0xbf,0xa9,0xf3,0x70,0xd6,0xf0,
  0xca,0x89,0xcb,0xc9,0x82,0x9d,0x13,0x79,0x0a,0x0f,0x25,0x19,0x3e,0x47,0xa3,0xa8,
  0xf9,0x5e,0xe8,0xa1,0xb0,0x71,0x1d,0x8c,0xde,0x69,0xe7,0x7c,0x56,0x3f,0x90,0xa4,
  0xeb,0x45,0x59,0xf1,0x97,0x4c,0x08,0xa0,0xb8,0x4a,0x86,0xc8,0xcd,0x98,0x7d,0xfc,
  0xef,0x4d,0x83,0x7e,0xdc,0x66,0x2b,0x8e,0xe0,0xa7,0xd0,0xa2,0x88,0x5f,0x7f,0xd9,
  0x9b,0x78,0xd1,0x8b,0xc3,0x8f,0x2d,0xe6,0x18,0x27,0x2c,0x24,0x94,0xb7,0xce,0xbd,
  0x0d,0x04,0x1c,0x09,0x16,0x23,0x00,0x1e,0x1a,0x29,0x2e,0x15,0x01,0x10,0x2a,0x20,
  0xbe,0x31,0x43,0x58,0xc2,0xaa,0x1f,0xe5,0xc5,0x9e,0xcf,0xc6,0x68,0xb2,0x80,0xf4,
  0xf8,0x53,0xb6,0x93,0x76,0x37,0x11,0x40,0xda,0x51,0xba,0x46,0x42,0x30,0x60,0x6d,
  0x5c,0x39,0x9f,0x48,0x6c,0x62,0x28,0x67,0x06,0x12,0x26,0x0e,0x33,0x50,0xa6,0x63,
  0xdd,0x3b,0xab,0x4b,0x72,0x5b,0x22,0x6f,0xb4,0x61,0x92,0x99,0x36,0x38,0x65,0xac,
  0x4f,0x2f,0x32,0x44,0x54,0x3c,0x03,0x5d,0x73,0x3a,0x77,0x84,0x8d,0x4e,0x49,0xd2,
  0xfb,0x91,0x6a,0xcc,0x8a,0x35,0x02,0x55,0x7a,0x34,0x96,0x3d,0xd3,0x41,0x85,0xf2,
  0xb1,0x75,0xc4,0xb5,0xbb,0xb3,0x1b,0xd5,0x07,0x05,0x17,0x0b,0x7b,0xd7,0xdf,0xea,
  0xe3,0x57,0xc0,0x95,0x9c,0x6e,0x14,0xae,0xb9,0x6b,0xc1,0x81,0x87,0x74,0xd8,0xe2,
  0xec,0x52,0xbc,0xe9,0xe1,0xdb,0x0c,0xf7,0xaf,0x5a,0x9a,0xc7,0xfa,0xf6,0xee,0xfe };

__host__ __device__ __forceinline__ uint32_t rc4(uint32_t x) {
  uint32_t y = 0;
  for (int i = 0; i < 4; i++) {
    y = (y << 2) | (3u - (x & 3u));
    x >>= 2;
  }
  return y;
}

// ---------------------------------------------------------------------------
// Extraction.  One CTA = EXT_TILE consecutive syncmer offsets j of one contig;
// each thread owns EXT_PER consecutive offsets and walks them with rolling
// 80-bit forward and reverse-complement k-mer registers and a five-wide
// window of canonical 8-mer hashes.  The selection is the closed (12,8)
// syncmer rule: j is kept iff the first of the five 8-mer hashes of the
// 12-mer at j is a minimum or the last one is (src/extract.c:168-196).
// ---------------------------------------------------------------------------

struct K80 {
  uint64_t hi;  // bases 0..31, base 0 in bits 63..62
  uint32_t lo;  // bases 32..39 in bits 15..0
};

__device__ __forceinline__ void k80_push_back(K80 &k, uint32_t b) {  // forward: shift left
  k.hi = (k.hi << 2) | (k.lo >> 14);
  k.lo = ((k.lo << 2) | b) & 0xffffu;
}
__device__ __forceinline__ void k80_push_front(K80 &k, uint32_t b) {  // reverse complement
  k.lo = (k.lo >> 2) | ((uint32_t)(k.hi & 3u) << 14);
  k.hi = (k.hi >> 2) | ((uint64_t)b << 62);
}

__device__ __forceinline__ uint32_t hash8(uint32_t qa, uint32_t qb, const uint8_t *tm,
                                          const uint8_t *tmrc) {
  uint32_t f = ((uint32_t)tm[qa] << 8) | tm[qb];
  uint32_t r = ((uint32_t)tmrc[qb] << 8) | tmrc[qa];
  return f < r ? f : r;
}

template <int MODE>
__global__ void __launch_bounds__(EXT_THREADS)
k_extract(const uint8_t *__restrict__ bps, const int64_t *__restrict__ clen,
          const int64_t *__restrict__ boff, const int32_t *__restrict__ tile_ctg,
          const int64_t *__restrict__ tile_j0, int ctgb, uint32_t *__restrict__ counts,
          const uint64_t *__restrict__ offsets, Rec *__restrict__ out,
          uint32_t *__restrict__ hist, uint32_t *__restrict__ cursor, int dshift) {
  __shared__ uint8_t s[EXT_SPAN];
  __shared__ uint8_t tm[256], tmrc[256];
  const int tid = threadIdx.x;
  const int ctg = tile_ctg[blockIdx.x];
  const int64_t j0 = tile_j0[blockIdx.x];
  const int64_t len = clen[ctg];
  const uint8_t *cb = bps + boff[ctg];
  const int64_t xs = j0 - EXT_LEFT;  // contig position of s[0]; a multiple of 4

  tm[tid] = c_tmap[tid];
  tmrc[tid] = c_tmap[rc4(tid)];
  for (int k = tid; k < EXT_SPAN / 4; k += EXT_THREADS) {
    int64_t x = xs + 4 * (int64_t)k;
    uint32_t b = (x >= 0 && x < len) ? cb[x >> 2] : 0u;
#pragma unroll
    for (int q = 0; q < 4; q++) s[4 * k + q] = (x + q >= 0 && x + q < len) ? ((b >> (2 * q)) & 3u) : 0;
  }
  __syncthreads();

  const int64_t jlast = len - TMER;  // last 12-mer offset
  const int64_t ja = j0 + (int64_t)tid * EXT_PER;
  const int64_t jb = min(ja + EXT_PER, jlast + 1);
  uint32_t nrec = 0;
  uint64_t woff = 0;
  if (MODE == EXT_WRITE) woff = offsets[(int64_t)blockIdx.x * EXT_THREADS + tid];
  const uint64_t strand_bit = (uint64_t)1 << (8 * ctgb - 1);

  if (ja < jb) {
    const uint8_t *p = s + (ja - xs);  // p[i] = base ja + i
    K80 fw = {0, 0}, rc = {0, 0};
    for (int i = 0; i < 40; i++) k80_push_back(fw, p[i]);
    for (int i = -28; i < 12; i++) k80_push_front(rc, 3u - p[i]);
    uint32_t h0, h1, h2, h3;
    {
      uint32_t q[12];
      for (int i = 0; i < 11; i++) q[i] = (p[i] << 6) | (p[i + 1] << 4) | (p[i + 2] << 2) | p[i + 3];
      h0 = hash8(q[0], q[4], tm, tmrc);
      h1 = hash8(q[1], q[5], tm, tmrc);
      h2 = hash8(q[2], q[6], tm, tmrc);
      h3 = hash8(q[3], q[7], tm, tmrc);
    }
    for (int64_t j = ja; j < jb; j++) {
      uint32_t h4 = hash8((uint32_t)(fw.hi >> 48) & 0xffu, (uint32_t)(fw.hi >> 40) & 0xffu, tm, tmrc);
      uint32_t m03 = min(min(h0, h1), min(h2, h3));
      uint32_t m14 = min(min(h1, h2), min(h3, h4));
      if (h0 <= m14 || h4 <= m03) {
#pragma unroll
        for (int strand = 0; strand < 2; strand++) {
          bool ok = strand == 0 ? (j <= len - KMER) : (j >= KMER - TMER);
          if (!ok) continue;
          const K80 &k = strand == 0 ? fw : rc;
          uint64_t pos = strand == 0 ? (uint64_t)j : (uint64_t)(j + TMER);
          uint64_t cs = (uint64_t)ctg | (strand ? strand_bit : 0);
          if (MODE == EXT_COUNT) {
            nrec++;
          } else {
            Rec r;
            r.hi = k.hi;
            r.lo = ((uint64_t)k.lo << 48) | (cs << 32) | pos;
            if (MODE == EXT_WRITE) {
              out[woff++] = r;
            } else if (MODE == EXT_HIST) {
              atomicAdd(&hist[rec_prefix(r) >> dshift], 1u);
            } else {  // EXT_DIGIT
              uint32_t slot = atomicAdd(&cursor[rec_prefix(r) >> dshift], 1u);
              out[slot] = r;
            }
          }
        }
      }
      h0 = h1; h1 = h2; h2 = h3; h3 = h4;
      k80_push_back(fw, p[j - ja + 40]);
      k80_push_front(rc, 3u - p[j - ja + 12]);
    }
  }
  if (MODE == EXT_COUNT) counts[(int64_t)blockIdx.x * EXT_THREADS + tid] = nrec;
}

void launch_extract(int mode, int ntiles, cudaStream_t st, const uint8_t *bps, const int64_t *clen,
                    const int64_t *boff, const int32_t *tile_ctg, const int64_t *tile_j0, int ctgb,
                    uint32_t *counts, const uint64_t *offsets, Rec *out, uint32_t *hist, uint32_t *cursor,
                    int dshift) {
  if (ntiles <= 0) return;
  switch (mode) {
    case EXT_COUNT:
      k_extract<EXT_COUNT><<<ntiles, EXT_THREADS, 0, st>>>(bps, clen, boff, tile_ctg, tile_j0, ctgb, counts,
                                                           offsets, out, hist, cursor, dshift);
      break;
    case EXT_WRITE:
      k_extract<EXT_WRITE><<<ntiles, EXT_THREADS, 0, st>>>(bps, clen, boff, tile_ctg, tile_j0, ctgb, counts,
                                                           offsets, out, hist, cursor, dshift);
      break;
    case EXT_HIST:
      k_extract<EXT_HIST><<<ntiles, EXT_THREADS, 0, st>>>(bps, clen, boff, tile_ctg, tile_j0, ctgb, counts,
                                                          offsets, out, hist, cursor, dshift);
      break;
    default:
      k_extract<EXT_DIGIT><<<ntiles, EXT_THREADS, 0, st>>>(bps, clen, boff, tile_ctg, tile_j0, ctgb, counts,
                                                           offsets, out, hist, cursor, dshift);
  }
}

// ---------------------------------------------------------------------------
// Prefix histogram of records already in HBM (used when records come from
// the host instead of from extraction), and the scatter into buckets.
// ---------------------------------------------------------------------------

__global__ void k_prefix_hist(const Rec *__restrict__ rec, int64_t n, uint32_t *__restrict__ hist) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&hist[rec_prefix(rec[i])], 1u);
}

__global__ void k_prefix_scatter(const Rec *__restrict__ in, int64_t n, uint32_t *__restrict__ cursor,
                                 Rec *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    Rec r = in[i];
    uint32_t slot = atomicAdd(&cursor[rec_prefix(r)], 1u);
    out[slot] = r;
  }
}

// Exclusive scan of a digit's npfx (4..64) prefix counts by one warp.
__device__ __forceinline__ void warp_scan_prefixes(const uint32_t *cnt, uint32_t *off, uint32_t total, int npfx) {
  const int lane = threadIdx.x & 31;
  const int per = npfx > 32 ? 2 : 1;
  const int b = lane * per;
  const uint32_t c0 = b < npfx ? cnt[b] : 0u, c1 = per == 2 ? cnt[b + 1] : 0u;
  uint32_t x = c0 + c1;
  const uint32_t own = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  const uint32_t pre = x - own;
  if (b < npfx) off[b] = pre;
  if (per == 2) off[b + 1] = pre + c0;
  if (lane == 0) off[npfx] = total;
}

template <int CAP>
__global__ void __launch_bounds__(1024)
k_digit_sort(Rec *__restrict__ rec, const uint32_t *__restrict__ dstart, uint32_t *__restrict__ start,
             const uint32_t *__restrict__ list, uint32_t *__restrict__ qnext, uint32_t *__restrict__ qnext_count,
             int dshift) {
  const int npfx = 1 << dshift;
  const uint32_t pmask = (uint32_t)npfx - 1u;
  extern __shared__ Rec sa[];                              // CAP records
  uint16_t *sb = reinterpret_cast<uint16_t *>(sa + CAP);  // CAP record indices grouped by prefix
  __shared__ uint32_t soff[MAX_DIGIT_PREFIXES + 1], scur[MAX_DIGIT_PREFIXES];
  static_assert(CAP <= 65536, "16-bit record indices");
  const uint32_t d = list ? list[blockIdx.x] : blockIdx.x;
  const uint32_t ds = dstart[d], m = dstart[d + 1] - ds;
  if (m > (uint32_t)CAP) {
    if (threadIdx.x == 0) qnext[atomicAdd(qnext_count, 1u)] = d;
    return;
  }
  if (threadIdx.x < npfx) scur[threadIdx.x] = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
    const Rec r = rec[ds + i];
    sa[i] = r;
    atomicAdd(&scur[rec_prefix(r) & pmask], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 32) warp_scan_prefixes(scur, soff, m, npfx);
  __syncthreads();
  if (threadIdx.x < npfx) {
    start[(d << dshift) + threadIdx.x] = ds + soff[threadIdx.x];
    scur[threadIdx.x] = soff[threadIdx.x];
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x)
    sb[atomicAdd(&scur[rec_prefix(sa[i]) & pmask], 1u)] = (uint16_t)i;
  __syncthreads();
  // each record's rank among its prefix bucket (records are distinct)
  for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) {
    const Rec x = sa[sb[k]];
    const uint32_t q = rec_prefix(x) & pmask;
    const uint32_t gs = soff[q], ge = soff[q + 1];
    uint32_t rank = 0;
    for (uint32_t j = gs; j < ge; j++) rank += rec_less(sa[sb[j]], x) ? 1u : 0u;
    rec[ds + gs + rank] = x;
  }
}

template <int CAP>
cudaError_t launch_cap(int grid, int threads, cudaStream_t st, Rec *rec, const uint32_t *dstart, uint32_t *start,
                       const uint32_t *list, uint32_t *qnext, uint32_t *qnext_count, int dshift) {
  const size_t smem = (size_t)CAP * (sizeof(Rec) + sizeof(uint16_t));
  PGA_CUDA_TRY(cudaFuncSetAttribute(k_digit_sort<CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_digit_sort<CAP><<<grid, threads, smem, st>>>(rec, dstart, start, list, qnext, qnext_count, dshift);
  return cudaGetLastError();
}

cudaError_t launch_digit_sort(int cap, int grid, int threads, cudaStream_t st, Rec *rec, const uint32_t *dstart,
                              uint32_t *start, const uint32_t *list, uint32_t *qnext, uint32_t *qnext_count,
                              int dshift) {
  switch (cap) {
    case DS_CAP: return launch_cap<DS_CAP>(grid, threads, st, rec, dstart, start, list, qnext, qnext_count, dshift);
    case DS_CAP_MID: return launch_cap<DS_CAP_MID>(grid, threads, st, rec, dstart, start, list, qnext, qnext_count, dshift);
    default: return cudaErrorInvalidValue;
  }
}

__global__ void __launch_bounds__(BD_THREADS)
k_big_digit(Rec *__restrict__ rec, const uint32_t *__restrict__ dstart, uint32_t *__restrict__ start,
            const uint32_t *__restrict__ list, const int64_t *__restrict__ toff, Rec *__restrict__ tmp_all,
            uint32_t *__restrict__ qmed, uint32_t *__restrict__ qbig, uint32_t *__restrict__ qcount, int dshift) {
  const int npfx = 1 << dshift;
  const uint32_t pmask = (uint32_t)npfx - 1u;
  __shared__ uint32_t soff[MAX_DIGIT_PREFIXES + 1], scur[MAX_DIGIT_PREFIXES];
  const uint32_t d = list[blockIdx.x];
  const uint32_t ds = dstart[d], m = dstart[d + 1] - ds;
  Rec *tmp = tmp_all + toff[blockIdx.x];
  if (threadIdx.x < npfx) scur[threadIdx.x] = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < m; i += BD_THREADS)
    atomicAdd(&scur[rec_prefix(rec[ds + i]) & pmask], 1u);
  __syncthreads();
  if (threadIdx.x < 32) warp_scan_prefixes(scur, soff, m, npfx);
  __syncthreads();
  if (threadIdx.x < npfx) {
    start[(d << dshift) + threadIdx.x] = ds + soff[threadIdx.x];
    scur[threadIdx.x] = soff[threadIdx.x];
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < m; i += BD_THREADS) {
    const Rec r = rec[ds + i];
    tmp[atomicAdd(&scur[rec_prefix(r) & pmask], 1u)] = r;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < m; i += BD_THREADS) rec[ds + i] = tmp[i];
  if (threadIdx.x < npfx) {
    const uint32_t n = soff[threadIdx.x + 1] - soff[threadIdx.x];
    const uint32_t p = (d << dshift) + threadIdx.x;
    if (n > 1) {
      if (n <= BK_MEDIUM) qmed[atomicAdd(&qcount[0], 1u)] = p;
      else {
        qbig[atomicAdd(&qcount[1], 1u)] = p;
        atomicMax(&qcount[2], n);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Finishing sort of each prefix bucket, by (k-mer, contig|strand, position).
// Buckets of up to BK_SMALL records are sorted by one thread each; larger
// ones are queued and sorted by one CTA in shared memory (up to BK_MEDIUM)
// or by a batched global-memory bitonic network.
// ---------------------------------------------------------------------------

// One CTA per run of `bpc` consecutive prefixes: the run's records (a
// contiguous range after the scatter) are staged in shared memory and each
// record writes itself to bucket start + rank, its rank being the number of
// records of its bucket that order before it (records are distinct, so the
// ranks are a permutation).  Buckets larger than BK_RANK_MAX, and every
// bucket of a run that does not fit in shared memory, are queued for the
// CTA-per-bucket (<= BK_MEDIUM) or global bitonic sort instead.
__global__ void __launch_bounds__(BK_THREADS)
k_bucket_rank(Rec *__restrict__ rec, const uint32_t *__restrict__ start, int bpc, int cap,
              uint32_t *__restrict__ qmed, uint32_t *__restrict__ qbig, uint32_t *__restrict__ qcount) {
  extern __shared__ Rec sm_rec[];
  const uint32_t p0 = blockIdx.x * (uint32_t)bpc;
  const uint32_t a = start[p0], b = start[p0 + bpc];
  const uint32_t m = b - a;
  if (m == 0) return;
  const bool fits = m <= (uint32_t)cap;
  // queue the buckets this kernel does not rank
  for (uint32_t q = threadIdx.x; q < (uint32_t)bpc; q += BK_THREADS) {
    uint32_t p = p0 + q;
    uint32_t n = start[p + 1] - start[p];
    if (n <= 1) continue;
    if (fits && n <= BK_RANK_MAX) continue;
    if (n <= BK_MEDIUM) qmed[atomicAdd(&qcount[0], 1u)] = p;
    else {
      qbig[atomicAdd(&qcount[1], 1u)] = p;
      atomicMax(&qcount[2], n);
    }
  }
  if (!fits) return;
  for (uint32_t i = threadIdx.x; i < m; i += BK_THREADS) sm_rec[i] = rec[a + i];
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < m; i += BK_THREADS) {
    Rec x = sm_rec[i];
    uint32_t p = rec_prefix(x);
    uint32_t bs = start[p] - a, be = start[p + 1] - a;
    uint32_t n = be - bs;
    if (n <= 1 || n > BK_RANK_MAX) continue;
    uint32_t rank = 0;
    for (uint32_t j = bs; j < be; j++) rank += rec_less(sm_rec[j], x) ? 1u : 0u;
    rec[a + bs + rank] = x;
  }
}

__device__ __forceinline__ void cswap(Rec &x, Rec &y) {
  if (rec_less(y, x)) {
    Rec t = x;
    x = y;
    y = t;
  }
}

// Bitonic sort variant whose every compare is ascending (the first step of
// each merge mirrors within the block), so a length that is not a power of
// two behaves as if padded with +infinity.
__global__ void __launch_bounds__(BK_THREADS)
k_bucket_medium(Rec *__restrict__ rec, const uint32_t *__restrict__ start,
                const uint32_t *__restrict__ qmed) {
  __shared__ Rec v[BK_MEDIUM];
  uint32_t p = qmed[blockIdx.x];
  uint32_t a = start[p];
  uint32_t n = start[p + 1] - a;
  for (uint32_t i = threadIdx.x; i < n; i += BK_THREADS) v[i] = rec[a + i];
  uint32_t np2 = 1;
  while (np2 < n) np2 <<= 1;
  __syncthreads();
  for (uint32_t k = 2; k <= np2; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t t = threadIdx.x; t < np2 / 2; t += BK_THREADS) {
        uint32_t i, q;
        if (j == (k >> 1)) {  // mirrored compare inside the k-block
          uint32_t blk = (t / j) * k, off = t % j;
          i = blk + off;
          q = blk + k - 1 - off;
        } else {
          i = (t / j) * 2 * j + (t % j);
          q = i + j;
        }
        if (q < n) cswap(v[i], v[q]);
      }
      __syncthreads();
    }
  }
  for (uint32_t i = threadIdx.x; i < n; i += BK_THREADS) rec[a + i] = v[i];
}

// One compare step of the same network over every queued big bucket
// (grid.y = queue slot).
__global__ void k_bucket_big_step(Rec *__restrict__ rec, const uint32_t *__restrict__ start,
                                  const uint32_t *__restrict__ qbig, uint32_t k, uint32_t j) {
  uint32_t p = qbig[blockIdx.y];
  uint32_t a = start[p];
  uint32_t n = start[p + 1] - a;
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t i, q;
  if (j == (k >> 1)) {
    uint64_t blk = (t / (k >> 1)) * k;
    uint32_t off = (uint32_t)(t % (k >> 1));
    i = (uint32_t)(blk + off);
    q = (uint32_t)(blk + (k - 1 - off));
  } else {
    i = (uint32_t)((t / j) * 2 * j + (t % j));
    q = i + j;
  }
  if (q < n) {
    Rec x = rec[a + i], y = rec[a + q];
    if (rec_less(y, x)) {
      rec[a + i] = y;
      rec[a + q] = x;
    }
  }
}

// ---------------------------------------------------------------------------
// LCPs, k-mer table entries, reference-format sorted records, prefix table.
// ---------------------------------------------------------------------------

__global__ void k_lcp(const Rec *__restrict__ rec, int64_t n, uint8_t *__restrict__ lcp) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    lcp[i] = (uint8_t)(i == 0 ? 0 : kmer_lcp(rec[i - 1], rec[i]));
}

// Writes `nbytes` staged bytes to dst with consecutive threads storing
// consecutive bytes (so every warp store covers one 32-byte span).
__device__ __forceinline__ void store_staged(const uint8_t *__restrict__ src, uint8_t *__restrict__ dst,
                                             int nbytes) {
  for (int k = threadIdx.x; k < nbytes; k += blockDim.x) dst[k] = src[k];
}

// Entry layout (src/kmer_adapter.c:60-65): k-mer bytes 3..9, mask 0, LCP,
// position (posb bytes LE), contig|strand (ctgb bytes LE).  One CTA of
// OUT_THREADS builds OUT_THREADS entries in shared memory, then stores them.
__global__ void __launch_bounds__(OUT_THREADS)
k_entries(const Rec *__restrict__ rec, const uint8_t *__restrict__ lcp, int64_t n,
          int posb, int ctgb, uint8_t *__restrict__ ent) {
  __shared__ uint8_t buf[OUT_THREADS * 24];
  const int eb = 9 + posb + ctgb;
  for (int64_t i0 = (int64_t)blockIdx.x * OUT_THREADS; i0 < n; i0 += (int64_t)gridDim.x * OUT_THREADS) {
    int64_t i = i0 + threadIdx.x;
    if (i < n) {
      Rec r = rec[i];
      uint8_t *d = buf + threadIdx.x * eb;
#pragma unroll
      for (int b = 3; b < 8; b++) d[b - 3] = (uint8_t)(r.hi >> (56 - 8 * b));
      d[5] = (uint8_t)(r.lo >> 56);
      d[6] = (uint8_t)(r.lo >> 48);
      d[7] = 0;
      d[8] = lcp[i];
      uint64_t pos = r.lo & 0xffffffffu, cs = (r.lo >> 32) & 0xffffu;
      for (int b = 0; b < posb; b++) d[9 + b] = (uint8_t)(pos >> (8 * b));
      for (int b = 0; b < ctgb; b++) d[9 + posb + b] = (uint8_t)(cs >> (8 * b));
    }
    __syncthreads();
    int cnt = (int)min((int64_t)OUT_THREADS, n - i0);
    store_staged(buf, ent + i0 * eb, cnt * eb);
    __syncthreads();
  }
}

// Record layout (src/record.h:8-26): LCP, k-mer 10 bytes, mask 0, position,
// contig|strand.  lcp may be null (extraction order: LCP byte 0).
__global__ void __launch_bounds__(OUT_THREADS)
k_records_out(const Rec *__restrict__ rec, const uint8_t *__restrict__ lcp, int64_t n,
              int posb, int ctgb, uint8_t *__restrict__ out) {
  __shared__ uint8_t buf[OUT_THREADS * 24];
  const int rs = 12 + posb + ctgb;
  for (int64_t i0 = (int64_t)blockIdx.x * OUT_THREADS; i0 < n; i0 += (int64_t)gridDim.x * OUT_THREADS) {
    int64_t i = i0 + threadIdx.x;
    if (i < n) {
      Rec r = rec[i];
      uint8_t *d = buf + threadIdx.x * rs;
      d[0] = lcp ? lcp[i] : 0;
#pragma unroll
      for (int b = 0; b < 8; b++) d[1 + b] = (uint8_t)(r.hi >> (56 - 8 * b));
      d[9] = (uint8_t)(r.lo >> 56);
      d[10] = (uint8_t)(r.lo >> 48);
      d[11] = 0;
      uint64_t pos = r.lo & 0xffffffffu, cs = (r.lo >> 32) & 0xffffu;
      for (int b = 0; b < posb; b++) d[12 + b] = (uint8_t)(pos >> (8 * b));
      for (int b = 0; b < ctgb; b++) d[12 + posb + b] = (uint8_t)(cs >> (8 * b));
    }
    __syncthreads();
    int cnt = (int)min((int64_t)OUT_THREADS, n - i0);
    store_staged(buf, out + i0 * rs, cnt * rs);
    __syncthreads();
  }
}

// Host-format records (rs bytes) -> Rec (and their LCP bytes when lcp != null).
__global__ void k_records_in(const uint8_t *__restrict__ in, int64_t n, int posb, int ctgb,
                             Rec *__restrict__ rec, uint8_t *__restrict__ lcp) {
  const int rs = 12 + posb + ctgb;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t *s = in + i * rs;
    uint64_t hi = 0, pos = 0, cs = 0;
#pragma unroll
    for (int b = 0; b < 8; b++) hi = (hi << 8) | s[1 + b];
    uint64_t lo16 = ((uint64_t)s[9] << 8) | s[10];
    for (int b = 0; b < posb; b++) pos |= (uint64_t)s[12 + b] << (8 * b);
    for (int b = 0; b < ctgb; b++) cs |= (uint64_t)s[12 + posb + b] << (8 * b);
    Rec r;
    r.hi = hi;
    r.lo = (lo16 << 48) | (cs << 32) | pos;
    rec[i] = r;
    if (lcp) lcp[i] = s[0];
  }
}

// cum[p] = number of records with prefix <= p = start[p+1]; also the largest
// bucket (the longest prefix group, which sizes FastGA's merge cache).
__global__ void k_prefix_table(const uint32_t *__restrict__ start, int64_t *__restrict__ cum,
                               uint32_t *__restrict__ maxrun) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t best = 0;
  if (p < NPREFIX) {
    uint32_t e = start[p + 1];
    if (cum) cum[p] = (int64_t)e;
    best = e - start[p];
  }
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0 && best) atomicMax(maxrun, best);
}

// ---------------------------------------------------------------------------
// Union of two sorted indices whose records all differ (a resident target's
// and a query's: their contigs differ).  Each record goes to its rank in the
// union: its own index plus the number of the other index's records below
// it, which is the other index's prefix-table entry for its prefix plus a
// lower bound inside that prefix bucket.  The a side's contig|strand field
// is rewritten from width actgb to ctgb (the strand bit moves to the top of
// the wider field; (strand, contig, position) order is the same in both).
// ---------------------------------------------------------------------------

__device__ __forceinline__ Rec rec_widen(Rec r, uint32_t from_sign, uint32_t to_sign) {
  const uint64_t cs = (r.lo >> 32) & 0xffff;
  const uint64_t w = (cs & (from_sign - 1)) | ((cs & from_sign) ? to_sign : 0);
  r.lo = (r.lo & ~(0xffffull << 32)) | (w << 32);
  return r;
}

__global__ void k_union_rank(const Rec *__restrict__ a, const uint32_t *__restrict__ sa, int64_t na, int actgb,
                             const Rec *__restrict__ b, const uint32_t *__restrict__ sb, int64_t nb, int ctgb,
                             Rec *__restrict__ out) {
  const uint32_t fs = 1u << (8 * actgb - 1), ts = 1u << (8 * ctgb - 1);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na + nb;
       i += (int64_t)gridDim.x * blockDim.x) {
    const bool from_a = i < na;
    const Rec x = from_a ? rec_widen(a[i], fs, ts) : b[i - na];
    const uint32_t p = rec_prefix(x);
    uint32_t lo = from_a ? sb[p] : sa[p], hi = from_a ? sb[p + 1] : sa[p + 1];
    while (lo < hi) {
      const uint32_t m = lo + ((hi - lo) >> 1);
      const Rec y = from_a ? b[m] : rec_widen(a[m], fs, ts);
      if (rec_less(y, x))
        lo = m + 1;
      else
        hi = m;
    }
    out[(from_a ? i : i - na) + lo] = x;
  }
}

__global__ void k_add_prefix_tables(uint32_t *__restrict__ start, const uint32_t *__restrict__ other) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p <= NPREFIX;
       p += (int64_t)gridDim.x * blockDim.x)
    start[p] += other[p];
}

}  // namespace pga
