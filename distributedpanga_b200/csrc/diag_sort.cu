// Diagonal sort of a seed unit: seeds -> 128-bit keys -> stable LSD radix
// sort over the key bytes that differ, one launch per byte.
//
// Reference: reimport_thread (src/fastga_pipeline.c:1391-1450) and rmsd_sort
// (lib/RSDsort.c:292-377), which sorts each A-contig panel on the whole
// reimported record.  The key (seeds.cuh: seed_key) orders every panel at
// once, so sorting the keys gives the panels' records in the reference's
// order.
//
// Layout while sorting: the low 64 bits of each key in one array and the bits
// above them (T - 64 of them for a T-bit key, 0-8 bytes) in a second, so a
// pass moves 8 + HB bytes per key each way instead of 16 (HB = 1 for the
// 72-bit keys of two 1 Gbp genomes).  The last pass writes the 128-bit keys
// that the alignment reads.
//
// A pass is one launch of persistent CTAs that take 4096-key tiles in order
// from a counter.  A tile's keys are ranked stably in registers (warp
// match-any ranks, per-warp digit counts), the tile publishes its digit
// counts, and thread d walks back over the tiles before it until it meets
// one whose running total of digit d is final (decoupled look-back); the
// tile then reorders its keys by digit in shared memory and writes each
// digit's run to its place with coalesced stores.  Every tile publishes its
// counts before it waits, and only waits on tiles taken before it, so the
// waits end; each is still bounded (DSP_SPIN_LIMIT polls, then the error
// flag, which also stops every other tile).  The histogram of a pass's digit
// is counted during the pass before it (keys already in registers); the
// first pass's comes from the key-building kernel.
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"
#include "diag_sort.cuh"
#include "scan.cuh"

namespace pga {

namespace {

constexpr int DSP_WARPS = DSP_THREADS / 32;
constexpr unsigned long long LB_AGG = 1ull << 62;   // word holds this tile's count
constexpr unsigned long long LB_INC = 2ull << 62;   // word holds the running total through this tile
constexpr unsigned long long LB_VAL = (1ull << 62) - 1;
constexpr int DSP_SPIN_LIMIT = 1 << 22;
constexpr int DSP_WINDOW = 4;  // look-back words read per step
constexpr int KEY_GRID_PER_SM = 8;

// scratch layout inside `small`
constexpr size_t SM_HIST = 0;                                   // 18 x 256 u32: [p] pass p, [16] byte 0, [17] byte 1
constexpr size_t SM_DSTART = SM_HIST + 18 * 256 * 4;            // 16 x 256 u64
constexpr size_t SM_CTR = SM_DSTART + 16 * 256 * 8;             // 16 u32 tile counters
constexpr size_t SM_BITS = SM_CTR + 64;                         // OR lo, OR hi, AND lo, AND hi
constexpr size_t SM_ERR = SM_BITS + 32;                         // int
constexpr size_t SM_END = SM_ERR + 16;
static_assert(SM_END <= DIAG_SORT_SMALL, "scratch layout");

template <int HB> struct HiOf { using T = uint8_t; };
template <> struct HiOf<2> { using T = uint16_t; };
template <> struct HiOf<4> { using T = uint32_t; };
template <> struct HiOf<8> { using T = uint64_t; };

__device__ __forceinline__ uint32_t key_byte(uint64_t lo, uint64_t hi, int shift) {
  return (uint32_t)((shift < 64 ? (lo >> shift) : (hi >> (shift - 64))) & 0xffu);
}

__device__ __forceinline__ unsigned long long ld_word(const unsigned long long *p) {
  return *(const volatile unsigned long long *)p;
}
__device__ __forceinline__ void st_word(unsigned long long *p, unsigned long long v) {
  *(volatile unsigned long long *)p = v;
}

// Keys of the seeds (split layout), their bit summaries (OR and AND over all
// keys) and the histograms of key bytes 0 and 1.
template <int HB>
__global__ void __launch_bounds__(256)
k_seed_keys_split(const Seed *__restrict__ sd, int64_t n, SeedKeyLayout L, uint64_t *__restrict__ lo,
                  typename HiOf<HB>::T *__restrict__ hi, uint32_t *__restrict__ hist01,
                  unsigned long long *__restrict__ bits) {
  using H = typename HiOf<HB>::T;
  __shared__ uint32_t h[2][256];
  __shared__ unsigned long long sb[4];
  h[0][threadIdx.x] = h[1][threadIdx.x] = 0;
  if (threadIdx.x == 0) {
    sb[0] = sb[1] = 0;
    sb[2] = sb[3] = ~0ull;
  }
  __syncthreads();
  unsigned long long olo = 0, ohi = 0, alo = ~0ull, ahi = ~0ull;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const U128 k = seed_key(sd[i], L);
    lo[i] = k.lo;
    if (HB) hi[i] = (H)k.hi;
    olo |= k.lo;
    ohi |= k.hi;
    alo &= k.lo;
    ahi &= k.hi;
    atomicAdd(&h[0][k.lo & 0xffu], 1u);
    atomicAdd(&h[1][(k.lo >> 8) & 0xffu], 1u);
  }
  for (int o = 16; o > 0; o >>= 1) {
    olo |= __shfl_xor_sync(0xffffffffu, olo, o);
    ohi |= __shfl_xor_sync(0xffffffffu, ohi, o);
    alo &= __shfl_xor_sync(0xffffffffu, alo, o);
    ahi &= __shfl_xor_sync(0xffffffffu, ahi, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicOr(&sb[0], olo);
    atomicOr(&sb[1], ohi);
    atomicAnd(&sb[2], alo);
    atomicAnd(&sb[3], ahi);
  }
  __syncthreads();
  if (threadIdx.x < 2) atomicOr(&bits[threadIdx.x], sb[threadIdx.x]);
  else if (threadIdx.x < 4) atomicAnd(&bits[threadIdx.x], sb[threadIdx.x]);
  for (int b = 0; b < 2; b++)
    if (h[b][threadIdx.x]) atomicAdd(&hist01[b * 256 + threadIdx.x], h[b][threadIdx.x]);
}

// Histogram of one key byte (the first pass's, when it is not byte 0 or 1).
template <int HB>
__global__ void __launch_bounds__(256)
k_key_hist(const uint64_t *__restrict__ lo, const typename HiOf<HB>::T *__restrict__ hi, int64_t n, int shift,
           uint32_t *__restrict__ hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&h[key_byte(lo[i], HB ? (uint64_t)hi[i] : 0ull, shift)], 1u);
  __syncthreads();
  if (h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// Exclusive prefix sums of one pass's 256 digit counts.
__global__ void __launch_bounds__(256) k_digit_starts(const uint32_t *__restrict__ hist,
                                                      unsigned long long *__restrict__ dstart) {
  __shared__ unsigned long long s[256];
  s[threadIdx.x] = hist[threadIdx.x];
  __syncthreads();
  for (int o = 1; o < 256; o <<= 1) {
    const unsigned long long v = threadIdx.x >= o ? s[threadIdx.x - o] : 0ull;
    __syncthreads();
    s[threadIdx.x] += v;
    __syncthreads();
  }
  dstart[threadIdx.x] = s[threadIdx.x] - hist[threadIdx.x];
}

// One LSD pass over key byte `shift` (see the file comment).  Writes the split
// layout, or the 128-bit keys when LAST.  Counts key byte next_shift (>= 0)
// into next_hist for the following pass.
template <int HB, bool LAST>
__global__ void __launch_bounds__(DSP_THREADS, 4)
k_diag_pass(const uint64_t *__restrict__ lo_in, const typename HiOf<HB>::T *__restrict__ hi_in,
            uint64_t *__restrict__ lo_out, typename HiOf<HB>::T *__restrict__ hi_out, U128 *__restrict__ aos_out,
            int64_t n, int shift, int next_shift, const unsigned long long *__restrict__ dstart,
            unsigned long long *__restrict__ look, uint32_t *__restrict__ tile_ctr,
            uint32_t *__restrict__ next_hist, int *__restrict__ err) {
  using H = typename HiOf<HB>::T;
  extern __shared__ __align__(16) unsigned char dsp_smem[];
  uint64_t *slo = reinterpret_cast<uint64_t *>(dsp_smem);  // the tile reordered by digit
  H *shi = reinterpret_cast<H *>(slo + DSP_TILE);
  __shared__ uint32_t wcnt[DSP_WARPS][256];  // per-warp digit counts, then per-warp offsets in a digit
  __shared__ uint32_t tst[256];              // tile-local start of each digit
  __shared__ unsigned long long gbase[256];  // global start of this tile's keys of each digit
  __shared__ uint32_t nh[256];               // next pass's digit counts
  __shared__ uint32_t scan_sm[33];
  __shared__ uint32_t s_tile;
  __shared__ int s_bad;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const int64_t ntiles = (n + DSP_TILE - 1) / DSP_TILE;
  nh[tid] = 0;
  if (tid == 0) s_bad = 0;
  for (;;) {
    if (tid == 0) s_tile = *(volatile int *)err ? 0xffffffffu : atomicAdd(tile_ctr, 1u);
#pragma unroll
    for (int w = 0; w < DSP_WARPS; w++) wcnt[w][tid] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    if ((int64_t)tile >= ntiles) break;
    // warp w holds keys [w * 512, w * 512 + 512) of the tile, 32 per round
    const int64_t wbase = (int64_t)tile * DSP_TILE + warp * (DSP_ITEMS * 32);
    // the keys' digits, four to a register (the keys themselves are read
    // again for the reorder, from cache, so that few registers stay live)
    uint32_t dig[DSP_ITEMS / 4];
#pragma unroll
    for (int q = 0; q < DSP_ITEMS / 4; q++) dig[q] = 0;
#pragma unroll
    for (int h0 = 0; h0 < DSP_ITEMS; h0 += DSP_ITEMS / 2) {  // two halves of loads in flight
      uint64_t klo[DSP_ITEMS / 2];
      H khi[DSP_ITEMS / 2];
#pragma unroll
      for (int j = 0; j < DSP_ITEMS / 2; j++) {
        const int64_t i = wbase + (h0 + j) * 32 + lane;
        klo[j] = 0;
        khi[j] = 0;
        if (i < n) {
          klo[j] = lo_in[i];
          if (HB) khi[j] = hi_in[i];
        }
      }
#pragma unroll
      for (int j = 0; j < DSP_ITEMS / 2; j++) {
        const int r = h0 + j;
        dig[r >> 2] |= key_byte(klo[j], (uint64_t)khi[j], shift) << (8 * (r & 3));
        if (next_shift >= 0 && wbase + r * 32 + lane < n)
          atomicAdd(&nh[key_byte(klo[j], (uint64_t)khi[j], next_shift)], 1u);
      }
    }
    // stable ranks: same-digit keys of earlier rounds, then of lower lanes
    // (16 bits each, two to a register)
    uint32_t rk[DSP_ITEMS / 2];
#pragma unroll
    for (int r = 0; r < DSP_ITEMS; r++) {
      const bool valid = wbase + r * 32 + lane < n;
      const uint32_t d = valid ? (dig[r >> 2] >> (8 * (r & 3))) & 0xffu : 256u + lane;
      const uint32_t m = __match_any_sync(0xffffffffu, d);
      const uint32_t pre = valid ? wcnt[warp][d] : 0u;
      const uint32_t rank = pre + __popc(m & lt);
      if (r & 1) rk[r >> 1] |= rank << 16;
      else rk[r >> 1] = rank;
      __syncwarp();
      if (valid && (m & lt) == 0) wcnt[warp][d] = pre + __popc(m);
      __syncwarp();
    }
    __syncthreads();
    // thread d: the tile's count of digit d and each warp's offset in it
    uint32_t cnt = 0;
#pragma unroll
    for (int w = 0; w < DSP_WARPS; w++) {
      const uint32_t c = wcnt[w][tid];
      wcnt[w][tid] = cnt;
      cnt += c;
    }
    // publish the count, then look back for the keys of digit d before this tile
    unsigned long long excl = 0;
    unsigned long long *mine = look + (size_t)tile * 256 + tid;
    if (tile == 0) {
      st_word(mine, LB_INC | cnt);
    } else {
      st_word(mine, LB_AGG | cnt);
      // DSP_WINDOW words of the tiles before t are read at once and used in
      // order: counts are added up to the first running total, or up to a
      // tile that has not published yet (read again from there)
      int64_t t = (int64_t)tile - 1;
      int spins = 0;
      bool ok = true;
      while (true) {
        unsigned long long v[DSP_WINDOW];
#pragma unroll
        for (int w = 0; w < DSP_WINDOW; w++) v[w] = t - w >= 0 ? ld_word(look + (size_t)(t - w) * 256 + tid) : 0ull;
        int used = 0;
        bool done = false;
#pragma unroll
        for (int w = 0; w < DSP_WINDOW; w++) {
          if (done || used < w) continue;
          const unsigned long long f = v[w] & ~LB_VAL;
          if (f == 0) continue;
          excl += v[w] & LB_VAL;
          used = w + 1;
          done = f == LB_INC;
        }
        if (done) break;
        t -= used;
        if (t < 0) {  // tile 0 always publishes its running total
          ok = false;
          break;
        }
        if (used == 0) {
          if (++spins > DSP_SPIN_LIMIT || *(volatile int *)err) {
            ok = false;
            break;
          }
          __nanosleep(64);
        }
      }
      if (ok) {
        st_word(mine, LB_INC | (excl + cnt));
      } else {
        atomicExch(err, 1);
        s_bad = 1;
      }
    }
    gbase[tid] = dstart[tid] + excl;
    tst[tid] = block_exclusive_scan<uint32_t>(cnt, scan_sm, nullptr);
    __syncthreads();
    if (s_bad) break;
    // the tile in digit order in shared memory
#pragma unroll 4
    for (int r = 0; r < DSP_ITEMS; r++) {
      const int64_t i = wbase + r * 32 + lane;
      if (i < n) {
        const uint32_t d = (dig[r >> 2] >> (8 * (r & 3))) & 0xffu;
        const uint32_t pos = tst[d] + wcnt[warp][d] + ((rk[r >> 1] >> (16 * (r & 1))) & 0xffffu);
        if (pos < (uint32_t)DSP_TILE) {
          slo[pos] = lo_in[i];
          if (HB) shi[pos] = hi_in[i];
        }
      }
    }
    __syncthreads();
    // each digit's run to its place
    const int64_t t0 = (int64_t)tile * DSP_TILE;
    const int tn = (int)((n - t0) < DSP_TILE ? (n - t0) : DSP_TILE);
    for (int j = tid; j < tn; j += DSP_THREADS) {
      const uint64_t l = slo[j];
      const uint64_t h = HB ? (uint64_t)shi[j] : 0ull;
      const uint32_t d = key_byte(l, h, shift);
      const unsigned long long o = gbase[d] + (unsigned long long)(j - (int)tst[d]);
      if (o < (unsigned long long)n) {
        if (LAST) {
          aos_out[o] = U128{l, h};
        } else {
          lo_out[o] = l;
          if (HB) hi_out[o] = (H)h;
        }
      }
    }
    __syncthreads();
  }
  __syncthreads();
  if (next_shift >= 0 && nh[tid]) atomicAdd(&next_hist[tid], nh[tid]);
}

}  // namespace

namespace {

int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

template <int HB, bool LAST>
cudaError_t launch_pass(const void *src, void *dst, int64_t n, int shift, int next_shift,
                        const unsigned long long *dstart, unsigned long long *look, uint32_t *ctr,
                        uint32_t *next_hist, int *err, cudaStream_t st) {
  using H = typename HiOf<HB>::T;
  const size_t dyn = (size_t)DSP_TILE * (8 + HB);
  auto kern = k_diag_pass<HB, LAST>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) return e;
  int occ = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, DSP_THREADS, dyn);
  if (e != cudaSuccess) return e;
  if (occ < 1) occ = 1;
  const int64_t ntiles = (n + DSP_TILE - 1) / DSP_TILE;
  const int grid = (int)(ntiles < (int64_t)sm_count() * occ ? ntiles : (int64_t)sm_count() * occ);
  const uint64_t *slo = (const uint64_t *)src;
  const H *shi = (const H *)(slo + n);
  uint64_t *dlo = (uint64_t *)dst;
  H *dhi = (H *)(dlo + n);
  kern<<<grid, DSP_THREADS, dyn, st>>>(slo, shi, dlo, dhi, (U128 *)dst, n, shift, next_shift, dstart, look, ctr,
                                       next_hist, err);
  return cudaGetLastError();
}

template <int HB>
cudaError_t sort_hb(void *a, void *b, int64_t n, const SeedKeyLayout &L, unsigned long long *look, char *sm,
                    cudaStream_t st, DiagSortResult *res) {
  using H = typename HiOf<HB>::T;
  uint32_t *hist = (uint32_t *)(sm + SM_HIST);
  unsigned long long *dstart = (unsigned long long *)(sm + SM_DSTART);
  uint32_t *ctr = (uint32_t *)(sm + SM_CTR);
  unsigned long long *bits = (unsigned long long *)(sm + SM_BITS);
  int *err = (int *)(sm + SM_ERR);
  cudaError_t e;
  if ((e = cudaMemsetAsync(sm, 0, SM_BITS, st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(bits, 0, 16, st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(bits + 2, 0xff, 16, st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(err, 0, 16, st)) != cudaSuccess) return e;
  // seeds (in a) -> split keys in b
  uint64_t *blo = (uint64_t *)b;
  const int64_t kb = (n + 255) / 256;
  const int kgrid = (int)(kb < (int64_t)sm_count() * KEY_GRID_PER_SM ? kb : (int64_t)sm_count() * KEY_GRID_PER_SM);
  k_seed_keys_split<HB><<<kgrid, 256, 0, st>>>((const Seed *)a, n, L, blo, (H *)(blo + n), hist + 16 * 256, bits);
  res->launches++;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  unsigned long long hb[4];
  if ((e = cudaMemcpyAsync(hb, bits, sizeof(hb), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  // the key bytes in which keys differ, least significant first
  int shifts[16], np = 0;
  const unsigned long long diff[2] = {hb[0] ^ hb[2], hb[1] ^ hb[3]};
  for (int byte = 0; byte < 8 + HB; byte++)
    if ((diff[byte >> 3] >> (8 * (byte & 7))) & 0xffull) shifts[np++] = 8 * byte;
  if (np == 0) shifts[np++] = 0;  // all keys equal: one pass writes the 128-bit keys
  // digit starts of the first pass
  const uint32_t *h0 = hist + 16 * 256;
  if (shifts[0] == 8) {
    h0 = hist + 17 * 256;
  } else if (shifts[0] != 0) {
    k_key_hist<HB><<<kgrid, 256, 0, st>>>(blo, (const H *)(blo + n), n, shifts[0], hist);
    res->launches++;
    h0 = hist;
  }
  k_digit_starts<<<1, 256, 0, st>>>(h0, dstart);
  res->launches++;
  void *src = b, *dst = a;
  const size_t lbytes = diag_sort_look_bytes(n);
  for (int p = 0; p < np; p++) {
    const bool last = p == np - 1;
    const int next = last ? -1 : shifts[p + 1];
    if ((e = cudaMemsetAsync(look, 0, lbytes, st)) != cudaSuccess) return e;
    e = last ? launch_pass<HB, true>(src, dst, n, shifts[p], next, dstart + 256 * p, look, ctr + p,
                                     hist + 256 * (p + 1), err, st)
             : launch_pass<HB, false>(src, dst, n, shifts[p], next, dstart + 256 * p, look, ctr + p,
                                      hist + 256 * (p + 1), err, st);
    if (e != cudaSuccess) return e;
    res->launches++;
    if (!last) {
      k_digit_starts<<<1, 256, 0, st>>>(hist + 256 * (p + 1), dstart + 256 * (p + 1));
      res->launches++;
    }
    void *t = src;
    src = dst;
    dst = t;
  }
  res->passes = np;
  res->in_a = src == a;
  int bad = 0;
  if ((e = cudaMemcpyAsync(&bad, err, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  res->bad = bad;
  return cudaGetLastError();
}

}  // namespace

cudaError_t diag_sort_seeds(void *a, void *b, int64_t n, const SeedKeyLayout &L, unsigned long long *look,
                            void *small, cudaStream_t st, DiagSortResult *res) {
  res->in_a = true;
  res->passes = 0;
  res->launches = 0;
  res->bad = 0;
  if (n <= 0) return cudaSuccess;
  const int T = L.total_bits;
  char *sm = (char *)small;
  if (T <= 64) return sort_hb<0>(a, b, n, L, look, sm, st, res);
  if (T <= 72) return sort_hb<1>(a, b, n, L, look, sm, st, res);
  if (T <= 80) return sort_hb<2>(a, b, n, L, look, sm, st, res);
  if (T <= 96) return sort_hb<4>(a, b, n, L, look, sm, st, res);
  return sort_hb<8>(a, b, n, L, look, sm, st, res);
}

}  // namespace pga
