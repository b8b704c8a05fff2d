// GDB ingest kernels: Create_GDB's FASTA reader (lib/GDB.c:771-1057) as
// tile-parallel passes over the text in HBM.
//
// The reader's line loop comes down to facts about each byte and each
// maximal run of N's (lib/GDB.c:850-977):
//   - a header line is a line whose first byte is '>'; its text after '>' and
//     any white space is the scaffold's name (lib/GDB.c:815-834);
//   - every other byte except '\n' is a sequence character, its value taken
//     from the reader's table (lib/GDB.c:350-367): A C G T (either case)
//     0..3, N/n 4 (not a base), any other character 0;
//   - the N runs of a scaffold join across line ends.  A run that ends the
//     scaffold is dropped; one shorter than nthr is filled with A's; any other
//     run ends the current contig and opens the next one, so a scaffold that
//     opens with such a run starts with an empty contig;
//   - each contig starts on a fresh byte of the 2-bit image, base i in bits
//     2*(i%4) of byte boff + i/4.
// So: find the headers, compact the sequence characters, find the runs,
// classify them, lay out the contigs and pack.  Every pass reads its input
// with 16-byte loads, one 4096-byte tile per 256-thread block.
#include <cstring>
#include "ingest.cuh"
#include "scan.cuh"

namespace pga {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int FA_BINS = FA_NSTATUS;   // 64 x 4 replicated base counters after the status words
constexpr int FA_NBINS = 64;

struct alignas(16) B16 {
  uint8_t b[16];
};

__device__ __forceinline__ B16 load16(const uint8_t *p, int64_t i0) {
  B16 r;
  *reinterpret_cast<uint4 *>(r.b) = __ldg(reinterpret_cast<const uint4 *>(p + i0));
  return r;
}

// The reader's base table (lib/GDB.c:350-367).
__device__ __forceinline__ uint32_t fa_value(uint32_t c) {
  const uint32_t l = c | 0x20u;
  return l == 'c' ? 1u : l == 'g' ? 2u : l == 't' ? 3u : l == 'n' ? 4u : 0u;
}

// isspace() of the C locale.
__device__ __forceinline__ bool fa_space(uint32_t c) {
  return c == ' ' || (c >= '\t' && c <= '\r');
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long y = __shfl_xor_sync(FULL, v, o);
    v = y < v ? y : v;
  }
  return v;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

// Last index j in [0, n) with a[j] <= x (a ascending, a[0] <= x).
__device__ __forceinline__ int64_t last_le(const int64_t *a, int64_t n, int64_t x) {
  int64_t lo = 0, hi = n;  // answer in [lo, hi)
  while (hi - lo > 1) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// First index j in [0, n) with a[j] >= x, or n.
__device__ __forceinline__ int64_t first_ge(const int64_t *a, int64_t n, int64_t x) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void k_init_status(unsigned long long *status) {
  for (int i = threadIdx.x; i < FA_NSTATUS + 4 * FA_NBINS; i += blockDim.x)
    status[i] = (i == FA_BAD || i == FA_EMPTY || i == FA_ALLN) ? ~0ull : 0ull;
}

// ---- headers ---------------------------------------------------------------

// Header starts of this thread's 16 bytes as a bit mask; NUL / non-ASCII
// bytes lower *bad.
__device__ __forceinline__ uint32_t header_bits(const uint8_t *text, int64_t n, int64_t i0,
                                                unsigned long long *bad) {
  if (i0 >= n) return 0;
  const B16 t = load16(text, i0);
  uint32_t prev = i0 > 0 ? text[i0 - 1] : '\n';
  uint32_t bits = 0;
  const int lim = n - i0 < FA_BYTES ? (int)(n - i0) : FA_BYTES;
#pragma unroll
  for (int k = 0; k < FA_BYTES; k++) {
    const uint32_t c = t.b[k];
    if (k < lim) {
      if ((c == 0 || c >= 128) && *bad == ~0ull) *bad = (unsigned long long)(i0 + k);
      if (c == '>' && prev == '\n') bits |= 1u << k;
    }
    prev = c;
  }
  return bits;
}

__global__ void __launch_bounds__(FA_THREADS) k_count_headers(const uint8_t *__restrict__ text, int64_t n,
                                                              int64_t *__restrict__ cnt,
                                                              unsigned long long *__restrict__ status) {
  __shared__ int64_t sm[33];
  const int64_t i0 = (int64_t)blockIdx.x * FA_TILE + (int64_t)threadIdx.x * FA_BYTES;
  unsigned long long bad = ~0ull;
  const uint32_t bits = header_bits(text, n, i0, &bad);
  int64_t tot;
  block_exclusive_scan<int64_t>(__popc(bits), sm, &tot);
  if (threadIdx.x == 0) cnt[blockIdx.x] = tot;
  bad = warp_min_u64(bad);
  if ((threadIdx.x & 31) == 0 && bad != ~0ull) atomicMin(&status[FA_BAD], bad);
}

__global__ void __launch_bounds__(FA_THREADS) k_write_headers(const uint8_t *__restrict__ text, int64_t n,
                                                              const int64_t *__restrict__ off,
                                                              int64_t *__restrict__ hstart) {
  __shared__ int64_t sm[33];
  const int64_t i0 = (int64_t)blockIdx.x * FA_TILE + (int64_t)threadIdx.x * FA_BYTES;
  unsigned long long bad = ~0ull;
  uint32_t bits = header_bits(text, n, i0, &bad);
  int64_t o = off[blockIdx.x] + block_exclusive_scan<int64_t>(__popc(bits), sm, (int64_t *)nullptr);
  while (bits) {
    const int k = __ffs(bits) - 1;
    bits &= bits - 1;
    hstart[o++] = i0 + k;
  }
}

// One warp per header line.  The text ends with '\n', so the search for the
// line end stops inside the text (the 64 zero bytes after it cover the last
// 32-byte step).
__global__ void k_header_lines(const uint8_t *__restrict__ text, const int64_t *__restrict__ hstart, int nh,
                               int64_t *__restrict__ hend, int64_t *__restrict__ htext,
                               int64_t *__restrict__ hlen1) {
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nh; j += nwarps) {
    const int64_t h = hstart[j];
    int64_t e = h + 1;
    for (int64_t b = h + 1;; b += 32) {
      const unsigned m = __ballot_sync(FULL, text[b + lane] == '\n');
      if (m) {
        e = b + __ffs(m) - 1;
        break;
      }
    }
    // for (s = 1; s < len; s++) if (!isspace(line[s])) break;   (lib/GDB.c:815-818)
    const int64_t len = e - h;
    int64_t s = len;
    for (int64_t b = h + 1; b < e; b += 32) {
      const int64_t i = b + lane;
      const unsigned m = __ballot_sync(FULL, i < e && !fa_space(text[i]));
      if (m) {
        s = b + __ffs(m) - 1 - h;
        break;
      }
    }
    if (lane == 0) {
      hend[j] = e;
      htext[j] = h + s;
      hlen1[j] = len - s + 1;
    }
  }
}

__global__ void k_copy_headers(const uint8_t *__restrict__ text, const int64_t *__restrict__ htext,
                               const int64_t *__restrict__ hlen1, const int64_t *__restrict__ hoff, int nh,
                               char *__restrict__ hdr) {
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nh; j += nwarps) {
    const int64_t src = htext[j], dst = hoff[j], len = hlen1[j] - 1;
    for (int64_t k = lane; k < len; k += 32) hdr[dst + k] = (char)text[src + k];
    if (lane == 0) hdr[dst + len] = '\0';
  }
}

// Marks [hstart, hend] (the header line and its '\n').
__global__ void k_paint_headers(const int64_t *__restrict__ hstart, const int64_t *__restrict__ hend, int nh,
                                uint32_t *__restrict__ mask) {
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nh; j += nwarps) {
    const int64_t a = hstart[j], b = hend[j];
    for (int64_t w = (a >> 5) + lane; w <= (b >> 5); w += 32) {
      const int64_t lo = a > (w << 5) ? a : (w << 5);
      const int64_t hi = b < (w << 5) + 31 ? b : (w << 5) + 31;
      const int nb = (int)(hi - lo + 1);
      const uint32_t m = (nb == 32 ? FULL : ((1u << nb) - 1u)) << (lo & 31);
      atomicOr(&mask[w], m);
    }
  }
}

// ---- sequence characters -----------------------------------------------------

// Sequence characters of this thread's 16 bytes as a bit mask.
__device__ __forceinline__ uint32_t seq_bits(const B16 &t, int64_t n, int64_t i0, const uint32_t *mask) {
  const uint32_t hm = (mask[i0 >> 5] >> (i0 & 31)) & 0xffffu;
  const int lim = n - i0 < FA_BYTES ? (int)(n - i0) : FA_BYTES;
  uint32_t bits = 0;
#pragma unroll
  for (int k = 0; k < FA_BYTES; k++)
    if (k < lim && t.b[k] != '\n') bits |= 1u << k;
  return bits & ~hm;
}

__global__ void __launch_bounds__(FA_THREADS) k_count_seq(const uint8_t *__restrict__ text, int64_t n,
                                                          const uint32_t *__restrict__ mask,
                                                          int64_t *__restrict__ cnt) {
  __shared__ int64_t sm[33];
  const int64_t i0 = (int64_t)blockIdx.x * FA_TILE + (int64_t)threadIdx.x * FA_BYTES;
  uint32_t bits = 0;
  if (i0 < n) bits = seq_bits(load16(text, i0), n, i0, mask);
  int64_t tot;
  block_exclusive_scan<int64_t>(__popc(bits), sm, &tot);
  if (threadIdx.x == 0) cnt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(FA_THREADS) k_write_seq(const uint8_t *__restrict__ text, int64_t n,
                                                          const uint32_t *__restrict__ mask,
                                                          const int64_t *__restrict__ off,
                                                          const int64_t *__restrict__ hend, int nh,
                                                          uint8_t *__restrict__ seq, int64_t *__restrict__ sstart,
                                                          unsigned long long *__restrict__ status) {
  __shared__ int64_t sm[33];
  __shared__ unsigned long long sbin[4];
  if (threadIdx.x < 4) sbin[threadIdx.x] = 0;
  const int64_t i0 = (int64_t)blockIdx.x * FA_TILE + (int64_t)threadIdx.x * FA_BYTES;
  B16 t;
  uint32_t bits = 0, hm = 0;
  if (i0 < n) {
    t = load16(text, i0);
    bits = seq_bits(t, n, i0, mask);
    hm = (mask[i0 >> 5] >> (i0 & 31)) & 0xffffu;
  }
  int64_t g = off[blockIdx.x] + block_exclusive_scan<int64_t>(__popc(bits), sm, (int64_t *)nullptr);
  uint32_t c4[4] = {0, 0, 0, 0};
  if (i0 < n) {
    const int lim = n - i0 < FA_BYTES ? (int)(n - i0) : FA_BYTES;
#pragma unroll
    for (int k = 0; k < FA_BYTES; k++) {
      if (k >= lim) break;
      const uint32_t c = t.b[k];
      if ((bits >> k) & 1u) {
        const uint32_t v = fa_value(c);
        seq[g++] = (uint8_t)v;
        if (v < 4) c4[v] += 1;
      } else if (((hm >> k) & 1u) && c == '\n') {
        // the '\n' of header line j: scaffold j's sequence starts here
        sstart[last_le(hend, nh, i0 + k)] = g;
      }
    }
  }
#pragma unroll
  for (int v = 0; v < 4; v++) {
    const uint32_t s = __reduce_add_sync(FULL, c4[v]);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(&sbin[v], (unsigned long long)s);
  }
  __syncthreads();
  if (threadIdx.x < 4 && sbin[threadIdx.x])
    atomicAdd(&status[FA_BINS + 4 * (blockIdx.x % FA_NBINS) + threadIdx.x], sbin[threadIdx.x]);
}

__global__ void k_flag_scaffolds(uint8_t *__restrict__ seq, const int64_t *__restrict__ sstart, int nh,
                                 unsigned long long *__restrict__ status) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nh; j += gridDim.x * blockDim.x) {
    const int64_t a = sstart[j], b = sstart[j + 1];
    if (a == b) atomicMin(&status[FA_EMPTY], (unsigned long long)j);
    else seq[a] |= 8;
  }
}

// ---- N runs ------------------------------------------------------------------

// Starts and ends (last N) of maximal N runs among this thread's 16 sequence
// positions; a scaffold's first position (bit 3) breaks a run.
__device__ __forceinline__ void run_bits(const uint8_t *seq, int64_t G, int64_t g0, uint32_t *sb, uint32_t *eb) {
  *sb = 0;
  *eb = 0;
  if (g0 >= G) return;
  const B16 t = load16(seq, g0);
  const uint32_t nxt16 = g0 + FA_BYTES < G ? seq[g0 + FA_BYTES] : 8u;
  uint32_t prev = g0 > 0 ? seq[g0 - 1] : 0u;
  const int lim = G - g0 < FA_BYTES ? (int)(G - g0) : FA_BYTES;
#pragma unroll
  for (int k = 0; k < FA_BYTES; k++) {
    const uint32_t x = t.b[k];
    const uint32_t nx = k + 1 < lim ? (uint32_t)t.b[k + 1 < FA_BYTES ? k + 1 : k] : (k + 1 == FA_BYTES ? nxt16 : 8u);
    if (k < lim && (x & 7u) == 4u) {
      if ((x & 8u) || g0 + k == 0 || (prev & 7u) != 4u) *sb |= 1u << k;
      if ((nx & 8u) || (nx & 7u) != 4u) *eb |= 1u << k;
    }
    prev = x;
  }
}

__global__ void __launch_bounds__(FA_THREADS) k_count_runs(const uint8_t *__restrict__ seq, int64_t G,
                                                           int64_t *__restrict__ cnt_start,
                                                           int64_t *__restrict__ cnt_end) {
  __shared__ int64_t sm[33];
  const int64_t g0 = (int64_t)blockIdx.x * FA_TILE + (int64_t)threadIdx.x * FA_BYTES;
  uint32_t sb, eb;
  run_bits(seq, G, g0, &sb, &eb);
  int64_t ts, te;
  block_exclusive_scan<int64_t>(__popc(sb), sm, &ts);
  block_exclusive_scan<int64_t>(__popc(eb), sm, &te);
  if (threadIdx.x == 0) {
    cnt_start[blockIdx.x] = ts;
    cnt_end[blockIdx.x] = te;
  }
}

__global__ void __launch_bounds__(FA_THREADS) k_write_runs(const uint8_t *__restrict__ seq, int64_t G,
                                                           const int64_t *__restrict__ off_start,
                                                           const int64_t *__restrict__ off_end,
                                                           int64_t *__restrict__ rs, int64_t *__restrict__ re) {
  __shared__ int64_t sm[33];
  const int64_t g0 = (int64_t)blockIdx.x * FA_TILE + (int64_t)threadIdx.x * FA_BYTES;
  uint32_t sb, eb;
  run_bits(seq, G, g0, &sb, &eb);
  int64_t os = off_start[blockIdx.x] + block_exclusive_scan<int64_t>(__popc(sb), sm, (int64_t *)nullptr);
  int64_t oe = off_end[blockIdx.x] + block_exclusive_scan<int64_t>(__popc(eb), sm, (int64_t *)nullptr);
  while (sb) {
    const int k = __ffs(sb) - 1;
    sb &= sb - 1;
    rs[os++] = g0 + k;
  }
  while (eb) {
    const int k = __ffs(eb) - 1;
    eb &= eb - 1;
    re[oe++] = g0 + k + 1;
  }
}

// A run that ends its scaffold is dropped (its length is the scaffold's
// trailing gap); one shorter than nthr is filled; any other splits.
__global__ void k_classify_runs(const int64_t *__restrict__ rs, const int64_t *__restrict__ re, int64_t R,
                                const int64_t *__restrict__ sstart, int nh, int nthr,
                                int64_t *__restrict__ is_split, int32_t *__restrict__ rscaf,
                                int64_t *__restrict__ trail, unsigned long long *__restrict__ status) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t r0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // every warp runs the same number of iterations so that the sums below see full warps
  const int64_t iters = (R + stride - 1) / stride;
  for (int64_t it = 0; it < iters; it++) {
    const int64_t r = r0 + it * stride;
    unsigned long long fill = 0;
    if (r < R) {
      const int64_t s = rs[r], e = re[r];
      const int j = (int)last_le(sstart, nh, s);
      const bool lead = s == sstart[j], tail = e == sstart[j + 1];
      int64_t split = 0;
      if (lead && tail) atomicMin(&status[FA_ALLN], (unsigned long long)j);
      else if (tail) trail[j] = e - s;
      else if (e - s < (int64_t)nthr) fill = (unsigned long long)(e - s);
      else split = 1;
      is_split[r] = split;
      rscaf[r] = j;
    }
    fill = warp_sum_u64(fill);
    if ((threadIdx.x & 31) == 0 && fill) atomicAdd(&status[FA_FILL], fill);
  }
}

// ---- contigs -------------------------------------------------------------------

__global__ void k_scaffolds(const int64_t *__restrict__ sstart, int nh, const int64_t *__restrict__ rs, int64_t R,
                            const int64_t *__restrict__ sr, int64_t nsplit, const int64_t *__restrict__ trail,
                            const int64_t *__restrict__ hoff, int64_t *__restrict__ scf4,
                            int64_t *__restrict__ cstart, int64_t *__restrict__ cend, int32_t *__restrict__ cscaf) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nh; j += gridDim.x * blockDim.x) {
    const int64_t a = sstart[j], b = sstart[j + 1];
    const int64_t q = first_ge(rs, R, a), q2 = first_ge(rs, R, b);
    const int64_t f = j + (q < R ? sr[q] : nsplit);
    const int64_t e = (j + 1) + (q2 < R ? sr[q2] : nsplit);
    scf4[4 * j + 0] = f;
    scf4[4 * j + 1] = e;
    scf4[4 * j + 2] = b - a - trail[j];
    scf4[4 * j + 3] = hoff[j];
    cstart[f] = a;
    cscaf[f] = j;
    cend[e - 1] = b - trail[j];
  }
}

__global__ void k_splits(const int64_t *__restrict__ rs, const int64_t *__restrict__ re, int64_t R,
                         const int64_t *__restrict__ is_split, const int64_t *__restrict__ sr,
                         const int32_t *__restrict__ rscaf, int64_t *__restrict__ cstart, int64_t *__restrict__ cend,
                         int32_t *__restrict__ cscaf) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < R; r += (int64_t)gridDim.x * blockDim.x) {
    if (!is_split[r]) continue;
    const int j = rscaf[r];
    const int64_t c = j + sr[r] + 1;
    cstart[c] = re[r];
    cend[c - 1] = rs[r];
    cscaf[c] = j;
  }
}

__global__ void k_contigs(int nc, const int64_t *__restrict__ cstart, const int64_t *__restrict__ cend,
                          const int32_t *__restrict__ cscaf, const int64_t *__restrict__ sstart,
                          int64_t *__restrict__ clen, int64_t *__restrict__ sbeg, int64_t *__restrict__ nbytes,
                          unsigned long long *__restrict__ status) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    const int64_t a = cstart[c], len = cend[c] - a;
    clen[c] = len;
    sbeg[c] = a - sstart[cscaf[c]];
    nbytes[c] = (len + 3) >> 2;
    atomicMax(&status[FA_MAXCTG], (unsigned long long)len);
  }
}

// One 4-byte word of the image per thread.
__global__ void k_pack(const uint8_t *__restrict__ seq, int nc, const int64_t *__restrict__ boff,
                       const int64_t *__restrict__ cstart, const int64_t *__restrict__ clen,
                       uint8_t *__restrict__ bps) {
  const int64_t total = boff[nc];
  const int64_t nwords = (total + 3) >> 2;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwords;
       w += (int64_t)gridDim.x * blockDim.x) {
    int64_t b = w << 2;
    int64_t c = last_le(boff, nc, b);
    uint32_t word = 0;
#pragma unroll
    for (int q = 0; q < 4; q++, b++) {
      if (b >= total) break;
      while (c + 1 < nc && boff[c + 1] <= b) c++;
      const int64_t i0 = (b - boff[c]) << 2, L = clen[c];
      const uint8_t *s = seq + cstart[c] + i0;
      uint32_t byte = 0;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        if (i0 + k < L) {
          const uint32_t v = s[k] & 7u;
          byte |= (v == 4u ? 0u : v) << (2 * k);
        }
      }
      word |= byte << (8 * q);
    }
    reinterpret_cast<uint32_t *>(bps)[w] = word;
  }
}

int grid_items(int64_t n, int threads, int cap = 148 * 16) {
  int64_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

unsigned tiles(int64_t n) { return (unsigned)((n + FA_TILE - 1) / FA_TILE); }

}  // namespace

cudaError_t fa_init_status(unsigned long long *status, cudaStream_t st) {
  k_init_status<<<1, 256, 0, st>>>(status);
  return cudaGetLastError();
}

cudaError_t fa_count_headers(const uint8_t *text, int64_t n, int64_t *cnt, unsigned long long *status,
                             cudaStream_t st) {
  k_count_headers<<<tiles(n), FA_THREADS, 0, st>>>(text, n, cnt, status);
  return cudaGetLastError();
}

cudaError_t fa_write_headers(const uint8_t *text, int64_t n, const int64_t *off, int64_t *hstart,
                             cudaStream_t st) {
  k_write_headers<<<tiles(n), FA_THREADS, 0, st>>>(text, n, off, hstart);
  return cudaGetLastError();
}

cudaError_t fa_header_lines(const uint8_t *text, const int64_t *hstart, int nh, int64_t *hend, int64_t *htext,
                            int64_t *hlen1, cudaStream_t st) {
  k_header_lines<<<grid_items((int64_t)nh * 32, 256), 256, 0, st>>>(text, hstart, nh, hend, htext, hlen1);
  return cudaGetLastError();
}

cudaError_t fa_copy_headers(const uint8_t *text, const int64_t *htext, const int64_t *hlen1, const int64_t *hoff,
                            int nh, char *hdr, cudaStream_t st) {
  k_copy_headers<<<grid_items((int64_t)nh * 32, 256), 256, 0, st>>>(text, htext, hlen1, hoff, nh, hdr);
  return cudaGetLastError();
}

cudaError_t fa_paint_headers(const int64_t *hstart, const int64_t *hend, int nh, uint32_t *mask, cudaStream_t st) {
  k_paint_headers<<<grid_items((int64_t)nh * 32, 256), 256, 0, st>>>(hstart, hend, nh, mask);
  return cudaGetLastError();
}

cudaError_t fa_count_seq(const uint8_t *text, int64_t n, const uint32_t *mask, int64_t *cnt, cudaStream_t st) {
  k_count_seq<<<tiles(n), FA_THREADS, 0, st>>>(text, n, mask, cnt);
  return cudaGetLastError();
}

cudaError_t fa_write_seq(const uint8_t *text, int64_t n, const uint32_t *mask, const int64_t *off,
                         const int64_t *hend, int nh, uint8_t *seq, int64_t *sstart,
                         unsigned long long *status, cudaStream_t st) {
  k_write_seq<<<tiles(n), FA_THREADS, 0, st>>>(text, n, mask, off, hend, nh, seq, sstart, status);
  return cudaGetLastError();
}

cudaError_t fa_flag_scaffolds(uint8_t *seq, const int64_t *sstart, int nh, unsigned long long *status,
                              cudaStream_t st) {
  k_flag_scaffolds<<<grid_items(nh, 256), 256, 0, st>>>(seq, sstart, nh, status);
  return cudaGetLastError();
}

cudaError_t fa_count_runs(const uint8_t *seq, int64_t G, int64_t *cnt_start, int64_t *cnt_end, cudaStream_t st) {
  k_count_runs<<<tiles(G), FA_THREADS, 0, st>>>(seq, G, cnt_start, cnt_end);
  return cudaGetLastError();
}

cudaError_t fa_write_runs(const uint8_t *seq, int64_t G, const int64_t *off_start, const int64_t *off_end,
                          int64_t *rs, int64_t *re, cudaStream_t st) {
  k_write_runs<<<tiles(G), FA_THREADS, 0, st>>>(seq, G, off_start, off_end, rs, re);
  return cudaGetLastError();
}

cudaError_t fa_classify_runs(const int64_t *rs, const int64_t *re, int64_t R, const int64_t *sstart, int nh,
                             int nthr, int64_t *is_split, int32_t *rscaf, int64_t *trail,
                             unsigned long long *status, cudaStream_t st) {
  k_classify_runs<<<grid_items(R, 256), 256, 0, st>>>(rs, re, R, sstart, nh, nthr, is_split, rscaf, trail, status);
  return cudaGetLastError();
}

cudaError_t fa_scaffolds(const int64_t *sstart, int nh, const int64_t *rs, int64_t R, const int64_t *sr,
                         int64_t nsplit, const int64_t *trail, const int64_t *hoff, int64_t *scf4,
                         int64_t *cstart, int64_t *cend, int32_t *cscaf, cudaStream_t st) {
  k_scaffolds<<<grid_items(nh, 256), 256, 0, st>>>(sstart, nh, rs, R, sr, nsplit, trail, hoff, scf4, cstart, cend,
                                                   cscaf);
  return cudaGetLastError();
}

cudaError_t fa_splits(const int64_t *rs, const int64_t *re, int64_t R, const int64_t *is_split, const int64_t *sr,
                      const int32_t *rscaf, int64_t *cstart, int64_t *cend, int32_t *cscaf, cudaStream_t st) {
  k_splits<<<grid_items(R, 256), 256, 0, st>>>(rs, re, R, is_split, sr, rscaf, cstart, cend, cscaf);
  return cudaGetLastError();
}

cudaError_t fa_contigs(int nc, const int64_t *cstart, const int64_t *cend, const int32_t *cscaf,
                       const int64_t *sstart, int64_t *clen, int64_t *sbeg, int64_t *nbytes,
                       unsigned long long *status, cudaStream_t st) {
  k_contigs<<<grid_items(nc, 256), 256, 0, st>>>(nc, cstart, cend, cscaf, sstart, clen, sbeg, nbytes, status);
  return cudaGetLastError();
}

cudaError_t fa_pack(const uint8_t *seq, int nc, const int64_t *boff, const int64_t *cstart, const int64_t *clen,
                    uint8_t *bps, cudaStream_t st) {
  k_pack<<<148 * 8, 256, 0, st>>>(seq, nc, boff, cstart, clen, bps);
  return cudaGetLastError();
}

}  // namespace pga
