// Seed reimport + diagonal sort that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host program that runs inside
// another framework's memory pool (PyTorch's caching allocator, a serving
// runtime's arena) owns all of the GPU memory it may use and must not
// allocate behind the pool's back, and a caller that has already reserved
// every byte its job is allowed would fail or evict the pool.  Such a caller
// hands in device buffers it already owns for the seeds and the sorted
// records; everything else this entry point needs lives in one file-scope
// device array of fixed size, compiled into the library.
//
// The array costs NOALLOC_SCRATCH_BYTES (about 12 MB) on every GPU that
// loads the library, for as long as the process lives.  Every call uses the
// same array, so calls whose work overlaps on the GPU (two host threads, or
// two streams) race and corrupt each other's results; the array keeps the
// last call's contents, and this code clears what must start at zero.
#include <cstdint>
#include <mutex>
#include <cuda.h>
#include <cuda_runtime.h>
#include "common.cuh"
#include "merge.cuh"
#include "radix.cuh"
#include "scan.cuh"
#include "seeds.cuh"
#include "../../include/pga_b200.h"

using namespace pga;

namespace {

constexpr int64_t NOALLOC_MAX_SEEDS = 1 << 18;  // 262,144 seeds per call
constexpr int64_t NB_MAX = (NOALLOC_MAX_SEEDS + RADIX_TILE - 1) / RADIX_TILE;
constexpr int64_t OFF_SEEDS = 0;
constexpr int64_t OFF_KEYS = OFF_SEEDS + NOALLOC_MAX_SEEDS * 16;
constexpr int64_t OFF_ALT = OFF_KEYS + NOALLOC_MAX_SEEDS * 16;
constexpr int64_t OFF_HIST = OFF_ALT + NOALLOC_MAX_SEEDS * 16;
constexpr int64_t OFF_SCAN = OFF_HIST + 256 * NB_MAX * 4;
constexpr int64_t OFF_ACC = OFF_SCAN + 4096;
constexpr int64_t NOALLOC_SCRATCH_BYTES = OFF_ACC + 256;

}  // namespace

// The scratch.  In host code this name is only a host-side stand-in for the
// symbol, never a device address: the address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int MAX_DEVICES = 128;
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
std::mutex g_setup_mu;
CtxGetCurrentFn g_ctx_get_current = nullptr;
CUcontext g_scratch_ctx[MAX_DEVICES] = {nullptr};
unsigned char *g_scratch_dev[MAX_DEVICES] = {nullptr};

// Device address of the scratch on the current device.  The address is
// looked up with that device current and kept with the context it belongs
// to; when the device's context is a different one (cudaDeviceReset and a
// new primary context load the module again, possibly elsewhere) it is
// looked up again.  The context comes from the driver's cuCtxGetCurrent,
// reached through the runtime so that the library needs no link to libcuda.
cudaError_t scratch_address(unsigned char **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
  e = cudaFree(nullptr);  // makes the device's primary context current
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (g_ctx_get_current == nullptr) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    e = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || fn == nullptr) return cudaErrorUnknown;
    g_ctx_get_current = (CtxGetCurrentFn)fn;
  }
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return cudaErrorUnknown;
  if (g_scratch_dev[dev] == nullptr || g_scratch_ctx[dev] != ctx) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_dev[dev] = (unsigned char *)p;
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_dev[dev];
  return cudaSuccess;
}

int grid1(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 32) g = 148 * 32;
  return (int)g;
}

int bitlen64(uint64_t v) {
  int b = 0;
  while (v) {
    b++;
    v >>= 1;
  }
  return b;
}

}  // namespace

extern "C" int pga_reimport_sort_noalloc(const uint8_t *seeds_dev, int64_t len, int position_bytes,
                                         int contig_strand_bytes, int comp, int ncontig, int64_t amxpos, int dbyte,
                                         uint8_t *out_dev, int64_t *panel_off_dev, void *stream) {
  const int posb = position_bytes, ctgb = contig_strand_bytes;
  if (len < 0 || (len > 0 && (!seeds_dev || !out_dev)) || !panel_off_dev || posb < 1 || posb > 4 || ctgb < 1 ||
      ctgb > 2 || (comp != 0 && comp != 1) || ncontig < 1 || ncontig > 32767 || dbyte < 1 || dbyte > 4 ||
      amxpos < 0)
    return PGA_ERR_ARG;
  const int sb = 1 + 2 * (posb + ctgb);
  if (len % sb != 0) return PGA_ERR_ARG;  // not a whole number of seeds
  const int64_t n = len / sb;
  if (n > NOALLOC_MAX_SEEDS) return PGA_ERR_LIMIT;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char *base = nullptr;
  if (scratch_address(&base) != cudaSuccess) return PGA_ERR_CUDA;
  Seed *sd = (Seed *)(base + OFF_SEEDS);
  U128 *keys = (U128 *)(base + OFF_KEYS);
  U128 *alt = (U128 *)(base + OFF_ALT);
  uint32_t *hist = (uint32_t *)(base + OFF_HIST);
  uint32_t *scan_tmp = (uint32_t *)(base + OFF_SCAN);
  unsigned long long *acc = (unsigned long long *)(base + OFF_ACC);

  // key layout: the same as pga_reimport_sort's (seeds.cuh)
  SeedKeyLayout L;
  L.comp = comp;
  L.amxpos = amxpos;
  L.bmxpos = amxpos;
  L.maxdag = 2 * amxpos;
  L.dbyte = dbyte;
  L.ctgb = ctgb;
  L.dmask = (1ull << (8 * dbyte)) - 1;
  L.jmask = (1ull << (8 * ctgb - 1)) - 1;
  uint64_t amax = (uint64_t)L.maxdag < L.dmask ? (uint64_t)L.maxdag : L.dmask;
  uint64_t bmax = (uint64_t)(L.maxdag >> 6) < L.dmask ? (uint64_t)(L.maxdag >> 6) : L.dmask;
  int wc = bitlen64((uint64_t)(ncontig > 1 ? ncontig - 1 : 1));
  L.off_dlow = 6;
  L.off_anti = 12;
  L.off_band = L.off_anti + bitlen64(amax);
  L.off_j = L.off_band + bitlen64(bmax);
  L.off_i = L.off_j + wc;
  L.w_i = wc;
  L.total_bits = L.off_i + wc;
  if (L.total_bits > 128) return PGA_ERR_LIMIT;

  U128 *res = keys;
  if (n > 0) {
    k_seeds_in<<<grid1(n), 256, 0, st>>>(seeds_dev, n, posb, ctgb, sd);
    k_seed_keys<<<grid1(n), 256, 0, st>>>(sd, n, L, keys);
    if (cudaMemsetAsync(acc, 0, 16, st) != cudaSuccess) return PGA_ERR_CUDA;  // left over from the last call
    k_u128_diffbits<<<grid1(n) < 148 * 4 ? grid1(n) : 148 * 4, 256, 0, st>>>(keys, n, acc);
    unsigned long long diff[2] = {0, 0};
    if (cudaMemcpyAsync(diff, acc, 16, cudaMemcpyDeviceToHost, st) != cudaSuccess) return PGA_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return PGA_ERR_CUDA;
    int passes[16], np = 0;
    for (int s = 0; s < 128; s += 8) {
      uint64_t w = s < 64 ? diff[0] : diff[1];
      if ((w >> (s & 63)) & 0xffull) passes[np++] = s;
    }
    if (radix_sort_u128(keys, alt, n, passes, np, hist, scan_tmp, &res, st) != cudaSuccess) return PGA_ERR_CUDA;
    k_seed_records<<<grid1(n), 256, 0, st>>>(res, n, L, out_dev);
  }
  k_panel_bounds<<<(ncontig + 1 + 255) / 256, 256, 0, st>>>(res, n, L, ncontig, panel_off_dev);
  if (cudaGetLastError() != cudaSuccess) return PGA_ERR_CUDA;
  return PGA_OK;
}
