// C-ABI layer: context, device buffers, stage drivers and the drop-in entry
// points declared in include/pga_b200.h.
#include <algorithm>
#include <cstdarg>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>

#include "common.cuh"
#include "index.cuh"
#include "merge.cuh"
#include "diag_sort.cuh"
#include "radix.cuh"
#include "scan.cuh"
#include "seeds.cuh"
#include "align.cuh"
#include "align_spec.h"
#include "ingest.cuh"
#include "arena.h"
#include "../../include/pga_b200.h"

using namespace pga;

namespace {

struct DBuf {
  void *p = nullptr;
  size_t cap = 0;
};

enum StageId {
  ST_EXTRACT_HIST, ST_SCAN, ST_EXTRACT_SCATTER, ST_BUCKET, ST_LCP, ST_ENTRIES, ST_MERGE, ST_DIAG, ST_ALIGN, ST_DIAG_C, ST_N
};

// the arena's driver calls (the context's timed cudaMalloc / cudaFree)
int arena_malloc(void *ctx, void **p, size_t bytes);
void arena_free(void *ctx, void *p);

}  // namespace

struct pga_ctx {
  int device = 0;
  cudaStream_t own = nullptr;
  cudaStream_t st = nullptr;
  char err[512] = {0};
  int64_t launches = 0;
  bool timing = false;
  cudaEvent_t ev[ST_N][2] = {};
  float stage_ms[ST_N] = {0};
  bool stage_used[ST_N] = {false};
  // host time inside cudaMalloc / cudaFree, per stage (slot ST_N: outside
  // every stage), since timing was last enabled
  int cur_stage = ST_N;
  int stage_prev[ST_N] = {0};
  double alloc_ms[ST_N + 1] = {0};
  int64_t alloc_calls = 0;
  int64_t sheds = 0;  // shed_align_buffers calls that freed something
  // every DBuf of the context lives in the arena
  Arena arena{arena_malloc, arena_free, this};

  // GDB
  bool have_gdb = false;
  int ncontig = 0;
  int64_t maxctg = 0;
  int64_t bps_bytes = 0;
  std::vector<int64_t> clen, boff;
  // GDB ingest (pga_gdb_ingest_fasta): the scaffold side of the GDB
  bool have_scaffolds = false;
  std::vector<int64_t> h_sbeg, h_scf4;   // per contig sbeg; per scaffold {fctg, ectg, slen, hoff}
  std::vector<int32_t> h_scaf;           // per contig
  std::vector<char> h_headers;
  int64_t base_count[4] = {0, 0, 0, 0};
  int ingest_nthr = 0;                   // the gap threshold the GDB was read with
  DBuf fa_text, fa_mask, fa_seq, fa_cnt, fa_tmp, fa_tot, fa_status, fa_hdr, fa_hbytes, fa_runs, fa_ctg;
  cudaEvent_t fa_ev[3] = {nullptr, nullptr, nullptr};  // upload start, parse start, parse end
  float ingest_ms[2] = {0, 0};                        // pga_gdb_ingest_times
  int posb = 0, ctgb = 0, rsize = 0;
  DBuf bps, dclen, dboff, tile_ctg, tile_j0;
  int ntiles = 0;
  std::vector<int32_t> h_tile_ctg;

  // index
  DBuf hist, start, scan_tmp, rec, rec2, lcp, ent, cum, qmed, qbig, qcount, maxrun, u64tmp, coarse;
  int64_t nrec = 0;
  bool have_index = false, have_entries = false;
  int64_t largest = 0;

  // merge
  DBuf blk_n, blk_c, blk_tmp, seed[2];
  int64_t nseed[2] = {0, 0};
  bool have_seeds = false;
  bool seeds_released = false;  // release_for_align freed the unsorted seeds
  bool seeds_loaded = false;    // the seeds came from pga_seeds_load, not pga_merge
  int freq = 0;

  // diagonal sort
  DBuf keys[2], dlook, dsmall, panel[2];
  U128 *sorted[2] = {nullptr, nullptr};
  bool seeds_consumed[2] = {false, false};  // the unit's seed buffer was used by its diagonal sort
  // served requests: the resident target whose recorded Local_Alignment
  // calls pga_align may use (set by pga_serve_load), the hit counter, and
  // the outcome for the last alignment: {used, calls answered from the
  // record, calls made, reason it was not used: 0 none, 1 no record,
  // 3 scoring tables differ}
  const pga_target *reuse_t = nullptr;
  DBuf memo_hits;
  int64_t reuse_stats[4] = {0, 0, 0, 0};
  // recording a target's own run (pga_target_create_reuse): the log of its
  // calls, sized for cap_calls calls and cap_bytes trace bytes
  bool capture = false;
  DBuf mlog_key, mlog_val, mlog_toff, mlog_trace, mlog_ctr;
  int64_t cap_calls = 0, cap_bytes = 0;
  // the scoring tables of the last alignment
  std::vector<int16_t> spec_host;
  int ave_path_host = 0;
  int diag_passes[2] = {0, 0};
  SeedKeyLayout lay[2];
  bool have_diag[2] = {false, false};

  // alignment
  float base_freq[4] = {.25f, .25f, .25f, .25f};
  bool freq_set = false;
  bool have_numeric = false;
  bool in_align = false;           // pga_align / pga_local_alignment hold the alignment buffers
  DBuf pk, poff, pwords;
  DBuf numf, numr, soff, spec_tab, tasks, task_next, pout, wave, points, cells, cell_next, ovl, perm, cand,
      cand_next, recs, rec_next, outb, out_next, pflag, pidx, pstart, pab, rng_ovl, rng_next, ftasks, fout,
      ridx, rout, selfb, pstart2, pab2, small, shist, fo_dev, binfo[2], plive[2];
  // survivors in la_sort order on the device (srecs, their traces in strace,
  // toff rewritten to offsets there), and their host copy, made when read
  DBuf srecs, slen, strace, skeys, skeys2, lhist, lscan;
  int64_t nalign = 0, ntrace = 0;
  bool host_valid = false;
  std::vector<AlnRec> h_recs;
  std::vector<uint8_t> h_trace;
  std::vector<int64_t> h_toff;     // offsets into h_trace
  int64_t align_stats[8] = {0};    // pga_align_stats
  float align_ms[4] = {0};         // pga_align_times
  int64_t align_work[4] = {0};     // pga_align_work
  int64_t align_prof[2] = {0};     // pga_align_profile: SM cycles in Local_Alignment, in finishing steps
  // pga_local_alignment: requests, paths, trace pool
  DBuf lreq, lpath, ltoff, ltrace, lnext;
  std::vector<int32_t> h_lpath;    // 7 ints per request
  std::vector<int64_t> h_ltoff;    // trace offsets in request order (n + 1)
  std::vector<uint16_t> h_ltrace;
  bool have_local = false;
  int64_t range_seeds = 0;         // pga_align_set_ranges
  int align_build = 0;             // pga_align_set_build: 0 by pair count, else 2..5 CTAs per SM
  int long_waves = -1;             // pga_align_set_long_waves: -1 automatic, 0 off, else the wave count
  int digit_bits = 0;              // pga_index_set_digit_bits: 0 by record count, else 18..22
  // pool use over the launches of one pga_align: candidate trace bytes,
  // range candidates, survivors, survivor trace bytes
  unsigned long long cand_used = 0, rng_used = 0, rec_used = 0, out_used = 0;
  unsigned long long counters[4] = {0, 0, 0, 0};  // staging for the device counters
  bool have_align = false;

  // generic byte staging
  DBuf io, io2;
};

// A resident target (pga_target_create): an ingested GDB and its sorted index,
// moved out of a context and kept on the device, read-only, for the requests
// of pga_serve_load on any context of the same device.
struct pga_target {
  int device = 0;
  int ncontig = 0, ctgb = 1, nthr = 0;
  int64_t bps_bytes = 0, nrec = 0;
  std::vector<int64_t> clen, boff, sbeg, scf4;
  std::vector<int32_t> scaf;
  std::vector<char> headers;
  int64_t base_count[4] = {0, 0, 0, 0};
  DBuf bps, rec, start;  // sequence image, sorted records, prefix table (NPREFIX + 1)
  // The target's own run's Local_Alignment calls (pga_target_create_reuse):
  // a table of their inputs and results (CallMemo), and the scoring tables
  // they were made with.
  struct Memo {
    bool valid = false;
    std::vector<int16_t> spec;
    int ave_path = 0;
    int64_t entries = 0, cap = 0;
    DBuf key, val, toff, trace;
  } memo;
};

namespace {

// Wave steps after which a call keeps its SM (pga_align_set_long_waves, automatic).
constexpr int LONG_WAVES_AUTO = 20000;

int fail(pga_ctx *c, int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(c->err, sizeof(c->err), fmt, ap);
  va_end(ap);
  return code;
}

#define CK(call)                                                                            \
  do {                                                                                      \
    cudaError_t _e = (call);                                                                \
    if (_e != cudaSuccess)                                                                  \
      return fail(ctx, PGA_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, \
                  __LINE__);                                                                \
  } while (0)

#define LAUNCHED(k) (ctx->launches += (k))

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Every device allocation and free of a context goes through these two, which
// charge their host time to the running stage.
cudaError_t dev_malloc(pga_ctx *ctx, void **p, size_t bytes) {
  const double t0 = now_ms();
  cudaError_t e = cudaMalloc(p, bytes);
  ctx->alloc_ms[ctx->cur_stage] += now_ms() - t0;
  ctx->alloc_calls++;
  return e;
}
void dev_free(pga_ctx *ctx, void *p) {
  if (!p) return;
  const double t0 = now_ms();
  cudaFree(p);
  ctx->alloc_ms[ctx->cur_stage] += now_ms() - t0;
  ctx->alloc_calls++;
}

int arena_malloc(void *ctx, void **p, size_t bytes) {
  if (dev_malloc((pga_ctx *)ctx, p, bytes) == cudaSuccess) return 0;
  cudaGetLastError();
  *p = nullptr;
  return 1;
}
void arena_free(void *ctx, void *p) { dev_free((pga_ctx *)ctx, p); }

// Frees the buffers only the alignment stage uses -- sequences, pools, task
// lists, local-alignment requests -- which the next pga_align or
// pga_local_alignment rebuilds, so that another stage can allocate.  Not while
// an alignment runs.  Returns whether anything was freed.
bool shed_align_buffers(pga_ctx *ctx) {
  if (ctx->in_align) return false;
  DBuf *bufs[] = {&ctx->numf, &ctx->numr, &ctx->pk, &ctx->wave, &ctx->points, &ctx->cells, &ctx->ovl, &ctx->perm,
                  &ctx->cand, &ctx->recs, &ctx->outb, &ctx->rng_ovl, &ctx->tasks, &ctx->pout, &ctx->pflag,
                  &ctx->pidx, &ctx->pstart, &ctx->pab, &ctx->pstart2, &ctx->pab2, &ctx->small, &ctx->ftasks,
                  &ctx->fout, &ctx->ridx, &ctx->rout, &ctx->lreq, &ctx->lpath, &ctx->ltoff, &ctx->ltrace,
                  &ctx->binfo[0], &ctx->binfo[1], &ctx->plive[0], &ctx->plive[1], &ctx->skeys, &ctx->skeys2,
                  &ctx->lhist, &ctx->lscan, &ctx->memo_hits, &ctx->mlog_key, &ctx->mlog_val, &ctx->mlog_toff,
                  &ctx->mlog_trace, &ctx->mlog_ctr};
  bool any = false;
  for (DBuf *b : bufs)
    if (b->p) {
      ctx->arena.release(b->p);
      b->p = nullptr;
      b->cap = 0;
      any = true;
    }
  ctx->have_numeric = false;
  if (any) ctx->sheds++;
  return any;
}

// Marks an alignment call for shed_align_buffers.
struct AlignScope {
  pga_ctx *c;
  explicit AlignScope(pga_ctx *x) : c(x) { c->in_align = true; }
  ~AlignScope() { c->in_align = false; }
};

// Grows b to at least `bytes` (contents not kept).  All of a context's work
// runs on its one stream, so a range freed here and handed out again is
// written only after the kernels that used it before.  Order of attempts: a
// range the arena holds; the same after shedding the last alignment's
// buffers (rebuilt by the next alignment); a new slab from the driver.
int ensure(pga_ctx *ctx, DBuf &b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.cap >= bytes) return PGA_OK;
  ctx->arena.release(b.p);
  b.p = nullptr;
  b.cap = 0;
  void *p = ctx->arena.fit(bytes);
  if (!p && shed_align_buffers(ctx)) p = ctx->arena.fit(bytes);
  if (!p) p = ctx->arena.alloc(bytes);
  if (!p)
    return fail(ctx, PGA_ERR_NOMEM, "device allocation of %zu bytes (context holds %zu, %zu of them free)", bytes,
                ctx->arena.held_bytes(), ctx->arena.free_bytes());
  b.p = p;
  b.cap = bytes;
  return PGA_OK;
}

// Grows b to `bytes`, keeping its first `keep` bytes.
int grow_keep(pga_ctx *ctx, DBuf &b, size_t bytes, size_t keep) {
  if (b.cap >= bytes) return PGA_OK;
  void *p = ctx->arena.alloc(bytes);
  if (!p)
    return fail(ctx, PGA_ERR_NOMEM, "device allocation of %zu bytes (context holds %zu, %zu of them free)", bytes,
                ctx->arena.held_bytes(), ctx->arena.free_bytes());
  if (keep > 0) {
    cudaError_t e = cudaMemcpyAsync(p, b.p, keep, cudaMemcpyDeviceToDevice, ctx->st);
    if (e != cudaSuccess) {
      ctx->arena.release(p);
      return fail(ctx, PGA_ERR_CUDA, "grow copy: %s", cudaGetErrorString(e));
    }
  }
  ctx->arena.release(b.p);
  b.p = p;
  b.cap = bytes;
  return PGA_OK;
}

#define ENSURE(b, bytes)                      \
  do {                                        \
    int _r = ensure(ctx, (b), (bytes));       \
    if (_r != PGA_OK) return _r;              \
  } while (0)

template <typename T>
T *P(DBuf &b) { return (T *)b.p; }
template <typename T>
const T *P(const DBuf &b) { return (const T *)b.p; }

int grid_for(int64_t n, int threads, int cap = 148 * 32) {
  int64_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

void stage_begin(pga_ctx *ctx, int s) {
  ctx->stage_prev[s] = ctx->cur_stage;
  ctx->cur_stage = s;
  if (ctx->timing) cudaEventRecord(ctx->ev[s][0], ctx->st);
}
void stage_end(pga_ctx *ctx, int s) {
  ctx->cur_stage = ctx->stage_prev[s];
  if (ctx->timing) {
    cudaEventRecord(ctx->ev[s][1], ctx->st);
    ctx->stage_used[s] = true;
  }
}

int bytes_inclusive(int64_t maxv) {
  int b = 0;
  int64_t cum = 1;
  while (cum < maxv + 1) {
    cum *= 256;
    b += 1;
  }
  return b;
}

int bitlen(uint64_t v) {
  int b = 0;
  while (v) {
    b++;
    v >>= 1;
  }
  return b;
}

// ---- index stages ---------------------------------------------------------

int sort_queued(pga_ctx *ctx);

// Prefixes per k_bucket_rank CTA: a power of two giving about BK_CAP/4
// records per CTA on average.
int bucket_run(const pga_ctx *ctx) {
  int bpc = 1;
  while (bpc < 4096 && (double)ctx->nrec * (bpc * 2) / NPREFIX <= BK_CAP / 4) bpc *= 2;
  return bpc;
}

// Buckets are already scattered by prefix into ctx->rec; `start` holds the
// exclusive scan (NPREFIX+1 entries).  Sort each bucket.
int sort_buckets(pga_ctx *ctx) {
  ENSURE(ctx->qmed, sizeof(uint32_t) * NPREFIX);
  ENSURE(ctx->qbig, sizeof(uint32_t) * NPREFIX);
  ENSURE(ctx->qcount, sizeof(uint32_t) * 4);
  CK(cudaMemsetAsync(ctx->qcount.p, 0, sizeof(uint32_t) * 4, ctx->st));
  const int bpc = bucket_run(ctx);
  CK(cudaFuncSetAttribute(k_bucket_rank, cudaFuncAttributeMaxDynamicSharedMemorySize, BK_CAP * (int)sizeof(Rec)));
  k_bucket_rank<<<NPREFIX / bpc, BK_THREADS, BK_CAP * sizeof(Rec), ctx->st>>>(
      P<Rec>(ctx->rec), P<uint32_t>(ctx->start), bpc, BK_CAP, P<uint32_t>(ctx->qmed), P<uint32_t>(ctx->qbig),
      P<uint32_t>(ctx->qcount));
  LAUNCHED(1);
  CK(cudaGetLastError());
  return sort_queued(ctx);
}

// The buckets k_bucket_rank / k_big_digit queued: one CTA each up to
// BK_MEDIUM records, the global bitonic network beyond.
int sort_queued(pga_ctx *ctx) {
  uint32_t q[4];
  CK(cudaMemcpyAsync(q, ctx->qcount.p, sizeof(q), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (q[0] > 0) {
    k_bucket_medium<<<q[0], BK_THREADS, 0, ctx->st>>>(P<Rec>(ctx->rec), P<uint32_t>(ctx->start),
                                                      P<uint32_t>(ctx->qmed));
    LAUNCHED(1);
    CK(cudaGetLastError());
  }
  if (q[1] > 0) {
    uint32_t np2 = 1;
    while (np2 < q[2]) np2 <<= 1;
    for (uint32_t k = 2; k <= np2; k <<= 1)
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        dim3 g((np2 / 2 + 255) / 256, q[1]);
        k_bucket_big_step<<<g, 256, 0, ctx->st>>>(P<Rec>(ctx->rec), P<uint32_t>(ctx->start),
                                                  P<uint32_t>(ctx->qbig), k, j);
        LAUNCHED(1);
      }
    CK(cudaGetLastError());
  }
  return PGA_OK;
}

// LCP bytes, optional entries, prefix table and the largest prefix group.
int finish_index(pga_ctx *ctx, bool want_entries) {
  int64_t n = ctx->nrec;
  ENSURE(ctx->lcp, (size_t)n + 16);
  stage_begin(ctx, ST_LCP);
  if (n > 0) {
    k_lcp<<<grid_for(n, 256), 256, 0, ctx->st>>>(P<Rec>(ctx->rec), n, P<uint8_t>(ctx->lcp));
    LAUNCHED(1);
  }
  stage_end(ctx, ST_LCP);
  stage_begin(ctx, ST_ENTRIES);
  ENSURE(ctx->maxrun, 16);
  CK(cudaMemsetAsync(ctx->maxrun.p, 0, 4, ctx->st));
  int64_t *cum = nullptr;
  if (want_entries) {
    int eb = 9 + ctx->posb + ctx->ctgb;
    ENSURE(ctx->ent, (size_t)n * eb + 16);
    ENSURE(ctx->cum, sizeof(int64_t) * NPREFIX);
    if (n > 0) {
      k_entries<<<grid_for(n, OUT_THREADS), OUT_THREADS, 0, ctx->st>>>(P<Rec>(ctx->rec), P<uint8_t>(ctx->lcp), n,
                                                                       ctx->posb, ctx->ctgb, P<uint8_t>(ctx->ent));
      LAUNCHED(1);
    }
    cum = P<int64_t>(ctx->cum);
  }
  k_prefix_table<<<NPREFIX / 256, 256, 0, ctx->st>>>(P<uint32_t>(ctx->start), cum, P<uint32_t>(ctx->maxrun));
  LAUNCHED(1);
  stage_end(ctx, ST_ENTRIES);
  CK(cudaGetLastError());
  uint32_t mr = 0;
  CK(cudaMemcpyAsync(&mr, ctx->maxrun.p, 4, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->largest = mr;
  ctx->have_index = true;
  ctx->have_entries = want_entries;
  ctx->have_seeds = false;
  ctx->have_diag[0] = ctx->have_diag[1] = false;
  return PGA_OK;
}

// hist (NPREFIX) -> start (NPREFIX+1, exclusive scan) and cursor = start.
int scan_hist(pga_ctx *ctx, int64_t *total) {
  ENSURE(ctx->scan_tmp, sizeof(uint32_t) * scan_tmp_elems(NPREFIX + 1));
  uint32_t *h = P<uint32_t>(ctx->hist), *s = P<uint32_t>(ctx->start);
  CK(cudaMemsetAsync(h + NPREFIX, 0, sizeof(uint32_t), ctx->st));
  CK(exclusive_scan<uint32_t>(h, s, NPREFIX + 1, P<uint32_t>(ctx->scan_tmp), (uint32_t *)nullptr, ctx->st));
  LAUNCHED(3);
  CK(cudaMemcpyAsync(h, s, sizeof(uint32_t) * NPREFIX, cudaMemcpyDeviceToDevice, ctx->st));  // cursor
  uint32_t t = 0;
  CK(cudaMemcpyAsync(&t, s + NPREFIX, 4, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  *total = t;
  return PGA_OK;
}

int check_records_fit(pga_ctx *ctx, int64_t n) {
  if (n >= (int64_t)0xffffffffLL)
    return fail(ctx, PGA_ERR_LIMIT, "%lld records: at most 2^32-2 supported", (long long)n);
  return PGA_OK;
}

// Host records (reference format) -> sorted device index (drop-in path).
int index_from_host(pga_ctx *ctx, const uint8_t *records, int64_t count, int posb, int ctgb) {
  int r = check_records_fit(ctx, count);
  if (r) return r;
  int rs = 12 + posb + ctgb;
  ctx->posb = posb;
  ctx->ctgb = ctgb;
  ctx->rsize = rs;
  ctx->nrec = count;
  ENSURE(ctx->io, (size_t)count * rs + 16);
  ENSURE(ctx->rec, sizeof(Rec) * (size_t)count + 16);
  ENSURE(ctx->rec2, sizeof(Rec) * (size_t)count + 16);
  ENSURE(ctx->hist, sizeof(uint32_t) * (NPREFIX + 1));
  ENSURE(ctx->start, sizeof(uint32_t) * (NPREFIX + 1));
  if (count > 0) {
    CK(cudaMemcpyAsync(ctx->io.p, records, (size_t)count * rs, cudaMemcpyHostToDevice, ctx->st));
    k_records_in<<<grid_for(count, 256), 256, 0, ctx->st>>>(P<uint8_t>(ctx->io), count, posb, ctgb, P<Rec>(ctx->rec2), nullptr);
    LAUNCHED(1);
  }
  CK(cudaMemsetAsync(ctx->hist.p, 0, sizeof(uint32_t) * NPREFIX, ctx->st));
  if (count > 0) {
    k_prefix_hist<<<grid_for(count, 256), 256, 0, ctx->st>>>(P<Rec>(ctx->rec2), count, P<uint32_t>(ctx->hist));
    LAUNCHED(1);
  }
  int64_t tot = 0;
  r = scan_hist(ctx, &tot);
  if (r) return r;
  if (count > 0) {
    k_prefix_scatter<<<grid_for(count, 256), 256, 0, ctx->st>>>(P<Rec>(ctx->rec2), count, P<uint32_t>(ctx->hist),
                                                                P<Rec>(ctx->rec));
    LAUNCHED(1);
  }
  CK(cudaGetLastError());
  return sort_buckets(ctx);
}

// Entries + prefix table (reference format, host) -> device records + LCPs.
__global__ void k_entries_in(const uint8_t *__restrict__ ent, const int64_t *__restrict__ cum, int64_t n,
                             int posb, int ctgb, Rec *__restrict__ rec, uint8_t *__restrict__ lcp) {
  const int eb = 9 + posb + ctgb;
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NPREFIX) return;
  int64_t a = p ? cum[p - 1] : 0, b = cum[p];
  if (b > n) b = n;
  for (int64_t i = a; i < b; i++) {
    const uint8_t *d = ent + i * eb;
    uint64_t hi = (uint64_t)p << 40;
    for (int k = 0; k < 5; k++) hi |= (uint64_t)d[k] << (32 - 8 * k);
    uint64_t lo16 = ((uint64_t)d[5] << 8) | d[6];
    uint64_t pos = 0, cs = 0;
    for (int k = 0; k < posb; k++) pos |= (uint64_t)d[9 + k] << (8 * k);
    for (int k = 0; k < ctgb; k++) cs |= (uint64_t)d[9 + posb + k] << (8 * k);
    Rec r;
    r.hi = hi;
    r.lo = (lo16 << 48) | (cs << 32) | pos;
    rec[i] = r;
    lcp[i] = d[8];
  }
}

// ---- merge ------------------------------------------------------------------

int run_merge(pga_ctx *ctx, int freq) {
  int64_t n = ctx->nrec;
  if (freq > MERGE_MAX_FREQ) return fail(ctx, PGA_ERR_LIMIT, "FREQ %d above %d", freq, MERGE_MAX_FREQ);
  int nb = (int)((n + MERGE_TILE - 1) / MERGE_TILE);
  if (nb < 1) nb = 1;
  ENSURE(ctx->blk_n, sizeof(uint32_t) * (nb + 1));
  ENSURE(ctx->blk_c, sizeof(uint32_t) * (nb + 1));
  ENSURE(ctx->blk_tmp, sizeof(uint32_t) * scan_tmp_elems(nb + 1) + 64);
  ENSURE(ctx->u64tmp, 64);
  stage_begin(ctx, ST_MERGE);
  uint32_t *bn = P<uint32_t>(ctx->blk_n), *bc = P<uint32_t>(ctx->blk_c);
  CK(cudaMemsetAsync(bn, 0, sizeof(uint32_t) * (nb + 1), ctx->st));
  CK(cudaMemsetAsync(bc, 0, sizeof(uint32_t) * (nb + 1), ctx->st));
  if (n > 0) {
    CK(launch_merge(false, nb, ctx->st, P<Rec>(ctx->rec), P<uint8_t>(ctx->lcp), n, freq, bn, bc, nullptr, nullptr,
                    ctx->ctgb));
    LAUNCHED(1);
  }
  uint32_t *tot = P<uint32_t>(ctx->u64tmp);
  CK(exclusive_scan<uint32_t>(bn, bn, nb + 1, P<uint32_t>(ctx->blk_tmp), tot, ctx->st));
  CK(exclusive_scan<uint32_t>(bc, bc, nb + 1, P<uint32_t>(ctx->blk_tmp), tot + 1, ctx->st));
  LAUNCHED(6);
  uint32_t t[2];
  CK(cudaMemcpyAsync(t, tot, 8, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->nseed[0] = t[0];
  ctx->nseed[1] = t[1];
  ENSURE(ctx->seed[0], sizeof(Seed) * (size_t)t[0] + 16);
  ENSURE(ctx->seed[1], sizeof(Seed) * (size_t)t[1] + 16);
  if (n > 0) {
    CK(launch_merge(true, nb, ctx->st, P<Rec>(ctx->rec), P<uint8_t>(ctx->lcp), n, freq, bn, bc,
                    P<Seed>(ctx->seed[0]), P<Seed>(ctx->seed[1]), ctx->ctgb));
    LAUNCHED(1);
  }
  stage_end(ctx, ST_MERGE);
  CK(cudaGetLastError());
  ctx->have_seeds = true;
  ctx->seeds_released = false;
  ctx->seeds_loaded = false;
  ctx->freq = freq;
  ctx->have_diag[0] = ctx->have_diag[1] = false;
  ctx->seeds_consumed[0] = ctx->seeds_consumed[1] = false;
  return PGA_OK;
}

// Per-A-contig seed counts of a device seed array (host result).
__global__ void k_seed_buck(const Seed *__restrict__ sd, int64_t n, unsigned long long *__restrict__ buck) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&buck[sd[i].b & 0xffffu], 1ull);
}

// ---- diagonal sort ------------------------------------------------------------

SeedKeyLayout make_layout(int comp, int ncontig, int64_t amxpos, int dbyte, int ctgb) {
  SeedKeyLayout L;
  L.comp = comp;
  L.amxpos = amxpos;
  L.bmxpos = amxpos;
  L.maxdag = 2 * amxpos;
  L.dbyte = dbyte;
  L.ctgb = ctgb;
  L.dmask = dbyte >= 8 ? ~0ull : ((1ull << (8 * dbyte)) - 1);
  L.jmask = (1ull << (8 * ctgb - 1)) - 1;
  uint64_t amax = std::min<uint64_t>((uint64_t)L.maxdag, L.dmask);
  uint64_t bmax = std::min<uint64_t>((uint64_t)(L.maxdag >> 6), L.dmask);
  int wc = bitlen((uint64_t)(ncontig > 1 ? ncontig - 1 : 1));
  L.off_dlow = 6;
  L.off_anti = 12;
  L.off_band = L.off_anti + bitlen(amax);
  L.off_j = L.off_band + bitlen(bmax);
  L.off_i = L.off_j + wc;
  L.w_i = wc;
  L.total_bits = L.off_i + wc;
  return L;
}

// Seeds of unit comp in ctx->seed[comp] -> sorted keys in ctx->keys[comp].
// The seed buffer is the sort's second buffer: the seeds are consumed.
int run_diag(pga_ctx *ctx, int comp, int ncontig, int64_t amxpos, int dbyte, int ctgb) {
  int64_t n = ctx->nseed[comp];
  SeedKeyLayout L = make_layout(comp, ncontig, amxpos, dbyte, ctgb);
  if (L.total_bits > 128) return fail(ctx, PGA_ERR_LIMIT, "diagonal sort key needs %d bits", L.total_bits);
  if (ctx->seeds_consumed[comp]) return fail(ctx, PGA_ERR_ARG, "the seeds of this unit were already sorted");
  ctx->lay[comp] = L;
  ENSURE(ctx->seed[comp], sizeof(Seed) * (size_t)n + 16);
  ENSURE(ctx->keys[comp], sizeof(U128) * (size_t)n + 16);
  ENSURE(ctx->dlook, diag_sort_look_bytes(n));
  ENSURE(ctx->dsmall, DIAG_SORT_SMALL);
  const int st_diag = comp ? ST_DIAG_C : ST_DIAG;
  stage_begin(ctx, st_diag);
  DiagSortResult R;
  CK(diag_sort_seeds(ctx->seed[comp].p, ctx->keys[comp].p, n, L, P<unsigned long long>(ctx->dlook),
                     ctx->dsmall.p, ctx->st, &R));
  LAUNCHED(R.launches);
  stage_end(ctx, st_diag);
  ctx->seeds_consumed[comp] = true;
  if (R.bad) return fail(ctx, PGA_ERR_CUDA, "diagonal sort: a pass stopped waiting for a tile before it");
  if (R.in_a) std::swap(ctx->seed[comp], ctx->keys[comp]);  // the keys ended in the seeds' buffer
  ctx->diag_passes[comp] = R.passes;
  ctx->sorted[comp] = P<U128>(ctx->keys[comp]);
  ctx->have_diag[comp] = true;
  return PGA_OK;
}

int copy_diag(pga_ctx *ctx, int comp, int ncontig, uint8_t *out, int64_t *panel_off) {
  int64_t n = ctx->nseed[comp];
  const SeedKeyLayout &L = ctx->lay[comp];
  int sw = 2 * L.dbyte + L.ctgb + 2;
  ENSURE(ctx->io, (size_t)n * sw + 16);
  ENSURE(ctx->panel[comp], sizeof(int64_t) * (ncontig + 1));
  if (n > 0) {
    k_seed_records<<<grid_for(n, 256), 256, 0, ctx->st>>>(ctx->sorted[comp], n, L, P<uint8_t>(ctx->io));
    LAUNCHED(1);
  }
  k_panel_bounds<<<(ncontig + 1 + 255) / 256, 256, 0, ctx->st>>>(ctx->sorted[comp], n, L, ncontig,
                                                                 P<int64_t>(ctx->panel[comp]));
  LAUNCHED(1);
  CK(cudaGetLastError());
  if (out && n > 0) CK(cudaMemcpyAsync(out, ctx->io.p, (size_t)n * sw, cudaMemcpyDeviceToHost, ctx->st));
  if (panel_off)
    CK(cudaMemcpyAsync(panel_off, ctx->panel[comp].p, sizeof(int64_t) * (ncontig + 1), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return PGA_OK;
}

int copy_seeds(pga_ctx *ctx, int comp, uint8_t *out, int64_t *buck) {
  int64_t n = ctx->nseed[comp];
  int sb = 1 + 2 * (ctx->posb + ctx->ctgb);
  if (out) {
    ENSURE(ctx->io, (size_t)n * sb + 16);
    if (n > 0) {
      k_seeds_out<<<grid_for(n, 256), 256, 0, ctx->st>>>(P<Seed>(ctx->seed[comp]), n, ctx->posb, ctx->ctgb,
                                                         P<uint8_t>(ctx->io));
      LAUNCHED(1);
      CK(cudaMemcpyAsync(out, ctx->io.p, (size_t)n * sb, cudaMemcpyDeviceToHost, ctx->st));
    }
  }
  if (buck) {
    ENSURE(ctx->io2, sizeof(uint64_t) * (ctx->ncontig + 1));
    CK(cudaMemsetAsync(ctx->io2.p, 0, sizeof(uint64_t) * ctx->ncontig, ctx->st));
    if (n > 0) {
      k_seed_buck<<<grid_for(n, 256), 256, 0, ctx->st>>>(P<Seed>(ctx->seed[comp]), n,
                                                         P<unsigned long long>(ctx->io2));
      LAUNCHED(1);
    }
    CK(cudaMemcpyAsync(buck, ctx->io2.p, sizeof(int64_t) * ctx->ncontig, cudaMemcpyDeviceToHost, ctx->st));
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  return PGA_OK;
}


// ---- alignment ------------------------------------------------------------------

// FastGA's order of contigs (the .gix permutation: longest first, equal
// lengths in contig order -- GIXmake's qsort on length, which glibc runs as a
// stable merge sort) and the self-pair entry rules of src/fastga_order_core.c.
struct FastgaOrder {
  int n = 0;
  std::vector<int> at, pos, range_start;
};

int64_t fo_key(int pos_b, int bepos) { return (((int64_t)(pos_b + 1)) << 32) | (uint32_t)bepos; }

// fo_compute_ranges (src/fastga_order_core.c:50-140) restated.
void fo_ranges(int n, const std::vector<int64_t> &clen_pos, int64_t npost, const std::vector<int64_t> &seeds,
               int64_t swide, int T, std::vector<int> &range_start) {
  std::vector<int> split(T + 1, 0);
  int p = 0, r = T;
  int64_t t = npost / T, cum = n > 0 ? clen_pos[0] : 0;
  for (int x = 1; x < n; x++) {
    if (cum >= t && x >= r) {
      p += 1;
      split[p] = x;
      t = (npost * (p + 1)) / T;
      r += T;
    }
    cum += clen_pos[x];
  }
  int nparts = p + 1;
  split[nparts] = n;
  range_start.resize(n);
  for (int x = 0; x < n; x++) range_start[x] = x;
  for (int i = 0; i < nparts; i++) {
    int64_t asize = 0;
    for (int x = split[i]; x < split[i + 1]; x++) asize += seeds[x] * swide;
    if (asize == 0) continue;
    int k = 0, beg, x;
    int64_t thr = asize / T, sum = 0;
    for (x = split[i]; x < split[i + 1]; x++)
      if (seeds[x] > 0) break;
    beg = x;
    for (; x < split[i + 1]; x++)
      if (seeds[x] > 0) {
        sum += seeds[x] * swide;
        if (sum >= thr) {
          for (int y = beg; y <= x; y++) range_start[y] = beg;
          k += 1;
          thr = (asize * (k + 1)) / T;
          beg = x + 1;
        }
      }
  }
}

// What one launch runs: tasks (whole pairs or band ranges, any order) and
// then the pairs to finish from their ranges (k_finish_pairs), each listing
// its range numbers, in order, at ridx[first .. first + nseg).
struct LaunchPlan {
  std::vector<PairTask> tasks;
  std::vector<FinishTask> fins;
  std::vector<int> ridx;
};

// Runs a plan: the warps take the tasks in plan order.  tout: one
// PairOut per task (plan order), fout: one per finished pair; rout_h (one
// per range number) is refreshed.  Pebbles live for one launch; candidate
// traces, range candidates and survivors accumulate over the launches of one
// pga_align.  A pool that overflows is grown (keeping what earlier launches
// left in it) and the launch runs again from the same counters.
int align_launch(pga_ctx *ctx, AlignLaunch &L, const LaunchPlan &plan, std::vector<PairOut> &tout,
                 std::vector<PairOut> &fout, std::vector<PairOut> &rout_h, long long *max_cycles,
                 int64_t *max_task_calls) {
  const size_t nt = plan.tasks.size(), nf = plan.fins.size();
  tout.assign(nt, PairOut{});
  fout.assign(nf, PairOut{});
  if (nt == 0 && nf == 0 && L.nsmall == 0) return PGA_OK;
  const std::vector<PairTask> &sorted = plan.tasks;  // the warps take them in this order
  if (nt) {
    ENSURE(ctx->tasks, sizeof(PairTask) * nt);
    ENSURE(ctx->pout, sizeof(PairOut) * nt);
    CK(cudaMemcpyAsync(ctx->tasks.p, sorted.data(), sizeof(PairTask) * nt, cudaMemcpyHostToDevice, ctx->st));
  }
  if (nf) {
    ENSURE(ctx->ftasks, sizeof(FinishTask) * nf);
    ENSURE(ctx->fout, sizeof(PairOut) * nf);
    ENSURE(ctx->ridx, sizeof(int) * (plan.ridx.size() + 1));
    CK(cudaMemcpyAsync(ctx->ftasks.p, plan.fins.data(), sizeof(FinishTask) * nf, cudaMemcpyHostToDevice, ctx->st));
    if (!plan.ridx.empty())
      CK(cudaMemcpyAsync(ctx->ridx.p, plan.ridx.data(), sizeof(int) * plan.ridx.size(), cudaMemcpyHostToDevice,
                         ctx->st));
  }
  std::vector<PairOut> ro(nt);
  const int grid = (int)((L.nwarps * 32 + ALIGN_THREADS - 1) / ALIGN_THREADS);
  const unsigned long long base[4] = {ctx->cand_used, ctx->rng_used, ctx->rec_used, ctx->out_used};
  for (int attempt = 0;; attempt++) {
    ctx->counters[0] = base[0];
    ctx->counters[1] = base[1];
    ctx->counters[2] = base[2];
    ctx->counters[3] = base[3];
    // the task counter, and the per-SM long-call flags after it
    CK(cudaMemsetAsync(ctx->task_next.p, 0, 64 + sizeof(unsigned) * aln::SM_FLAGS, ctx->st));
    L.smflag = P<unsigned>(ctx->task_next) + 16;
    L.prof = (unsigned long long *)(P<uint8_t>(ctx->task_next) + 32);
    // automatic: on for launches bounded by their longest calls, off for the
    // throughput-bound ones (the builds of three or more CTAs per SM), whose flagged SMs would
    // idle warps that still have queue work
    L.long_waves = ctx->long_waves >= 0 ? ctx->long_waves : (L.min_blocks >= 3 ? 0 : LONG_WAVES_AUTO);
    CK(cudaMemsetAsync(ctx->cell_next.p, 0, 8, ctx->st));
    CK(cudaMemcpyAsync(ctx->cand_next.p, &ctx->counters[0], 8, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->rng_next.p, &ctx->counters[1], 8, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->rec_next.p, &ctx->counters[2], 8, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->out_next.p, &ctx->counters[3], 8, cudaMemcpyHostToDevice, ctx->st));
    L.rout = P<PairOut>(ctx->rout);
    if (L.nsmall > 0) {
      // the device-planned pairs' reductions: sred[6] (first failing task) starts at ~0
      CK(cudaMemsetAsync(L.sred, 0, sizeof(unsigned long long) * (8 + 2 * (size_t)ctx->ncontig), ctx->st));
      CK(cudaMemsetAsync(L.sred + 6, 0xff, sizeof(unsigned long long), ctx->st));
    }
    if (nt || L.nsmall > 0) {
      L.tasks = P<PairTask>(ctx->tasks);
      L.ntasks = (int)nt;
      L.pout = P<PairOut>(ctx->pout);
      launch_align(L, grid, ctx->st);
      LAUNCHED(1);
      CK(cudaGetLastError());
      if (nt) CK(cudaMemcpyAsync(ro.data(), ctx->pout.p, sizeof(PairOut) * nt, cudaMemcpyDeviceToHost, ctx->st));
    }
    unsigned long long sred[8] = {0, 0, 0, 0, 0, 0, ~0ull, 0};
    if (L.nsmall > 0) CK(cudaMemcpyAsync(sred, L.sred, sizeof(sred), cudaMemcpyDeviceToHost, ctx->st));
    if (nf) {
      AlignLaunch F = L;
      F.ftasks = P<FinishTask>(ctx->ftasks);
      F.nftasks = (int)nf;
      F.range_idx = P<int>(ctx->ridx);
      F.pout = P<PairOut>(ctx->fout);
      launch_finish(F, grid, ctx->st);
      LAUNCHED(1);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(fout.data(), ctx->fout.p, sizeof(PairOut) * nf, cudaMemcpyDeviceToHost, ctx->st));
    }
    if (!rout_h.empty())
      CK(cudaMemcpyAsync(rout_h.data(), ctx->rout.p, sizeof(PairOut) * rout_h.size(), cudaMemcpyDeviceToHost,
                         ctx->st));
    unsigned long long used[4] = {0, 0, 0, 0}, prof[2] = {0, 0};
    CK(cudaMemcpyAsync(prof, L.prof, 16, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(&used[0], ctx->cand_next.p, 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(&used[1], ctx->rng_next.p, 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(&used[2], ctx->rec_next.p, 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(&used[3], ctx->out_next.p, 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    int errs = (int)sred[3], bad = -1, badf = -1;
    for (size_t k = 0; k < nt; k++)
      if (ro[k].err) {
        errs |= ro[k].err;
        if (bad < 0) bad = (int)k;
      }
    for (size_t f = 0; f < nf; f++)
      if (fout[f].err) {
        errs |= fout[f].err;
        if (badf < 0) badf = (int)f;
      }
    if (errs == 0) {
      ctx->align_prof[0] += (int64_t)prof[0];
      ctx->align_prof[1] += (int64_t)prof[1];
      ctx->cand_used = used[0];
      ctx->rng_used = used[1];
      ctx->rec_used = used[2];
      ctx->out_used = used[3];
      break;
    }
    // grow what overflowed and run the launch again
    bool grown = false;
    if (attempt < 6) {
      int r = PGA_OK;
      // pebble numbers are int: at most 2^31 - 1 pebbles
      const size_t max_cells = sizeof(aln::Pebble) * (size_t)0x7fffffff;
      if ((errs & aln::ALN_ERR_CELLS) && ctx->cells.cap < max_cells) {
        r = r ? r : ensure(ctx, ctx->cells, std::min(2 * ctx->cells.cap, max_cells));
        L.cell_cap = (int64_t)(ctx->cells.cap / sizeof(aln::Pebble));
        L.cells = P<aln::Pebble>(ctx->cells);
        grown = true;
      }
      if (errs & aln::ALN_ERR_TRACE) {
        r = r ? r : grow_keep(ctx, ctx->cand, 2 * ctx->cand.cap, base[0]);
        L.cand_cap = (int64_t)ctx->cand.cap;
        L.cand_bytes = P<uint8_t>(ctx->cand);
        grown = true;
      }
      if (errs & 0x800) {
        r = r ? r : grow_keep(ctx, ctx->rng_ovl, 2 * ctx->rng_ovl.cap, sizeof(aln::Ovl) * base[1]);
        L.rng_cap = (int64_t)(ctx->rng_ovl.cap / sizeof(aln::Ovl));
        L.rng_ovl = P<aln::Ovl>(ctx->rng_ovl);
        grown = true;
      }
      if (errs & 0x400) {
        r = r ? r : grow_keep(ctx, ctx->recs, 2 * ctx->recs.cap, sizeof(AlnRec) * base[2]);
        r = r ? r : grow_keep(ctx, ctx->outb, 2 * ctx->outb.cap, base[3]);
        L.rec_cap = (int64_t)(ctx->recs.cap / sizeof(AlnRec));
        L.out_cap = (int64_t)ctx->outb.cap;
        L.recs = P<AlnRec>(ctx->recs);
        L.out_bytes = P<uint8_t>(ctx->outb);
        grown = true;
      }
      if ((errs & 0x1000) || ((errs & aln::ALN_ERR_OVLS) && !(errs & (0x400 | 0x800)))) {
        int64_t oc = 2 * L.ovl_cap;
        r = r ? r : ensure(ctx, ctx->ovl, sizeof(aln::Ovl) * (size_t)L.nwarps * oc);
        r = r ? r : ensure(ctx, ctx->perm, sizeof(int) * 2 * (size_t)L.nwarps * oc);
        L.ovl_cap = oc;
        L.ovl = P<aln::Ovl>(ctx->ovl);
        L.perm = P<int>(ctx->perm);
        grown = true;
      }
      if (r) return r;
    }
    if (!grown) {
      if (sred[3])
        return fail(ctx, PGA_ERR_LIMIT, "alignment of a contig pair overflowed its work space (err 0x%llx)", sred[3]);
      if (bad >= 0)
        return fail(ctx, PGA_ERR_LIMIT, "alignment of pair (%d,%d,%s) overflowed its work space (err 0x%x)",
                    sorted[bad].a, sorted[bad].b, sorted[bad].comp ? "C" : "N", ro[bad].err);
      return fail(ctx, PGA_ERR_LIMIT, "alignment of pair (%d,%d,%s) overflowed its work space (err 0x%x)",
                  plan.fins[badf].a, plan.fins[badf].b, plan.fins[badf].comp ? "C" : "N", fout[badf].err);
    }
  }
  for (size_t k = 0; k < nt; k++) {
    tout[k] = ro[k];
    ctx->align_work[0] += ro[k].waves;
    ctx->align_work[1] += ro[k].cells;
    ctx->align_work[3] += 1;
    if (ro[k].cycles > *max_cycles) {
      *max_cycles = ro[k].cycles;
      *max_task_calls = ro[k].calls;
    }
  }
  if (L.nsmall > 0) {
    unsigned long long sred[8];
    CK(cudaMemcpyAsync(sred, L.sred, sizeof(sred), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->align_work[0] += (int64_t)sred[4];
    ctx->align_work[1] += (int64_t)sred[5];
    ctx->align_work[3] += L.nsmall;
    if ((long long)(sred[2] >> 16) > *max_cycles) {
      *max_cycles = (long long)(sred[2] >> 16);
      *max_task_calls = (int64_t)(sred[2] & 0xffff);
    }
  }
  return PGA_OK;
}

// Calls and exit bepos of a pair run as ranges: the sum, and the last range
// (in order) that called, else `entry`.
void combine_ranges(const std::vector<PairOut> &rout_h, const std::vector<int> &ids, int *calls, int *exit_bepos,
                    int entry) {
  *calls = 0;
  *exit_bepos = entry;
  for (int id : ids) {
    *calls += rout_h[id].calls;
    if (rout_h[id].calls > 0) *exit_bepos = rout_h[id].exit_bepos;
  }
}

// NUMERIC (with sentinels) and 2-bit packed copies of every contig, the base
// frequencies if not given, and the scoring tables (New_Align_Spec).
int prepare_sequences(pga_ctx *ctx, int *ave_path) {
  const int nc = ctx->ncontig;
  if (!ctx->have_numeric) {
    std::vector<int64_t> so(nc + 1);
    int64_t o = 1;
    for (int c = 0; c < nc; c++) {
      so[c] = o;
      o += ctx->clen[c] + 1;
    }
    so[nc] = o;
    ENSURE(ctx->numf, o + 16);
    ENSURE(ctx->numr, o + 16);
    ENSURE(ctx->soff, sizeof(int64_t) * (nc + 1));
    CK(cudaMemcpyAsync(ctx->soff.p, so.data(), sizeof(int64_t) * (nc + 1), cudaMemcpyHostToDevice, ctx->st));
    launch_numeric(P<uint8_t>(ctx->bps), P<int64_t>(ctx->dclen), P<int64_t>(ctx->dboff), P<int64_t>(ctx->soff), nc,
                   P<uint8_t>(ctx->numf), P<uint8_t>(ctx->numr), ctx->st);
    LAUNCHED(1);
    std::vector<int64_t> po(nc + 1), pw(nc + 1);
    int64_t wsum = 0;
    for (int c = 0; c < nc; c++) {
      pw[c] = ctx->clen[c] / 32 + 2;
      po[c] = wsum;
      wsum += pw[c];
    }
    ENSURE(ctx->pk, sizeof(uint64_t) * 4 * (size_t)(wsum + 1));
    ENSURE(ctx->poff, sizeof(int64_t) * (nc + 1));
    ENSURE(ctx->pwords, sizeof(int64_t) * (nc + 1));
    CK(cudaMemcpyAsync(ctx->poff.p, po.data(), sizeof(int64_t) * (nc + 1), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->pwords.p, pw.data(), sizeof(int64_t) * (nc + 1), cudaMemcpyHostToDevice, ctx->st));
    launch_pack(P<uint8_t>(ctx->numf), P<int64_t>(ctx->soff), P<int64_t>(ctx->dclen), P<int64_t>(ctx->poff),
                P<int64_t>(ctx->pwords), nc, P<uint64_t>(ctx->pk), ctx->st);
    LAUNCHED(1);
    if (!ctx->freq_set) {
      ENSURE(ctx->u64tmp, 64);
      CK(cudaMemsetAsync(ctx->u64tmp.p, 0, 32, ctx->st));
      launch_base_counts(P<uint8_t>(ctx->bps), P<int64_t>(ctx->dclen), P<int64_t>(ctx->dboff), nc,
                         P<unsigned long long>(ctx->u64tmp), ctx->st);
      LAUNCHED(1);
      unsigned long long cnt[4];
      CK(cudaMemcpyAsync(cnt, ctx->u64tmp.p, 32, cudaMemcpyDeviceToHost, ctx->st));
      CK(cudaStreamSynchronize(ctx->st));
      unsigned long long tot = cnt[0] + cnt[1] + cnt[2] + cnt[3];
      for (int q = 0; q < 4; q++) ctx->base_freq[q] = tot ? (float)((1. * cnt[q]) / tot) : .25f;
    }
    ctx->have_numeric = true;
  }
  std::vector<int16_t> tab(2 * 32768);
  *ave_path = aln::build_align_spec(ctx->base_freq, tab.data(), tab.data() + 32768);
  ENSURE(ctx->spec_tab, sizeof(int16_t) * tab.size());
  CK(cudaMemcpyAsync(ctx->spec_tab.p, tab.data(), sizeof(int16_t) * tab.size(), cudaMemcpyHostToDevice, ctx->st));
  ctx->spec_host.swap(tab);  // (a pageable source is staged before the copy call returns)
  ctx->ave_path_host = *ave_path;

  return PGA_OK;
}

// The aligner's launch description and work spaces (pools sized from the
// input; align_launch grows one that overflows).
int prepare_workspace(pga_ctx *ctx, AlignLaunch &L, int ave_path) {
  memset(&L, 0, sizeof(L));
  L.keysN = ctx->sorted[0];
  L.keysC = ctx->sorted[1];
  L.layN = ctx->lay[0];
  L.layC = ctx->lay[1];
  for (int comp = 0; comp < 2; comp++) {
    // the units' band info: which band blocks can hold a chain that passes the hit test
    const int64_t n = ctx->nseed[comp];
    ENSURE(ctx->binfo[comp], sizeof(uint16_t) * (size_t)n + 16);
    launch_band_info(ctx->sorted[comp], n, ctx->lay[comp], P<uint16_t>(ctx->binfo[comp]), ctx->st);
    LAUNCHED(n > 0 ? 1 : 0);
  }
  CK(cudaGetLastError());
  L.infoN = P<uint16_t>(ctx->binfo[0]);
  L.infoC = P<uint16_t>(ctx->binfo[1]);
  L.fwd = P<uint8_t>(ctx->numf);
  L.rc = P<uint8_t>(ctx->numr);
  L.soff = P<int64_t>(ctx->soff);
  L.clen = P<int64_t>(ctx->dclen);
  L.pk = P<uint64_t>(ctx->pk);
  L.poff = P<int64_t>(ctx->poff);
  L.pwords = P<int64_t>(ctx->pwords);
  L.score = P<int16_t>(ctx->spec_tab);
  L.table = P<int16_t>(ctx->spec_tab) + 32768;
  L.ave_path = ave_path;
  L.amxpos = ctx->maxctg;
  L.maxdag = 2 * ctx->maxctg;
  L.nwarps = 148 * 20;  // work spaces for the five-CTA build's resident warps
  L.vcap = 8192;
  L.point_cap = 4 * (ctx->maxctg / 100 + 4) + 64;
  // Pools sized from the sequence total; align_run_tasks grows one that
  // overflows and reruns the launch.  Buffers keep their size across calls.
  int64_t seqtot = 0;
  for (int c = 0; c < ctx->ncontig; c++) seqtot += ctx->clen[c];
  ENSURE(ctx->task_next, 64 + sizeof(unsigned) * aln::SM_FLAGS);
  ENSURE(ctx->wave, sizeof(int) * (size_t)L.nwarps * L.vcap * WAVE_INTS);
  ENSURE(ctx->points, sizeof(uint16_t) * (size_t)L.nwarps * L.point_cap);
  ENSURE(ctx->ovl, sizeof(aln::Ovl) * (size_t)L.nwarps * 16384);
  ENSURE(ctx->perm, sizeof(int) * 2 * (size_t)L.nwarps * 16384);
  ENSURE(ctx->rng_ovl, sizeof(aln::Ovl) * (size_t)std::max<int64_t>(1 << 18, seqtot / 256));
  {
    // 4 pebbles per input base to start, within what pebble numbers (int)
    // address and a third of the free memory; an overflow grows the pool
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    int64_t want = std::max<int64_t>(1 << 24, 4 * seqtot);
    want = std::min<int64_t>(want, 0x7fffffff);
    const int64_t have = (int64_t)((free_b + ctx->cells.cap) / 3 / sizeof(aln::Pebble));
    want = std::max<int64_t>(1 << 24, std::min(want, have));
    ENSURE(ctx->cells, sizeof(aln::Pebble) * (size_t)want);
  }
  ENSURE(ctx->cand, (size_t)std::max<int64_t>(64 << 20, 2 * seqtot));
  ENSURE(ctx->recs, sizeof(AlnRec) * (size_t)std::max<int64_t>(1 << 20, seqtot / 256));
  ENSURE(ctx->outb, (size_t)std::max<int64_t>(64 << 20, seqtot / 8));
  L.ovl_cap = (int64_t)(ctx->ovl.cap / (sizeof(aln::Ovl) * L.nwarps));
  L.rng_cap = (int64_t)(ctx->rng_ovl.cap / sizeof(aln::Ovl));
  L.cell_cap = (int64_t)(ctx->cells.cap / sizeof(aln::Pebble));
  L.cand_cap = (int64_t)ctx->cand.cap;
  L.rec_cap = (int64_t)(ctx->recs.cap / sizeof(AlnRec));
  L.out_cap = (int64_t)ctx->outb.cap;
  ENSURE(ctx->rng_next, 64);
  ENSURE(ctx->cell_next, 64);
  ENSURE(ctx->cand_next, 64);
  ENSURE(ctx->rec_next, 64);
  ENSURE(ctx->out_next, 64);
  L.next_task = P<unsigned>(ctx->task_next);
  L.wave = P<int>(ctx->wave);
  L.points = P<uint16_t>(ctx->points);
  L.ovl = P<aln::Ovl>(ctx->ovl);
  L.perm = P<int>(ctx->perm);
  L.cells = P<aln::Pebble>(ctx->cells);
  L.cell_next = P<unsigned long long>(ctx->cell_next);
  L.cand_bytes = P<uint8_t>(ctx->cand);
  L.cand_next = P<unsigned long long>(ctx->cand_next);
  L.recs = P<AlnRec>(ctx->recs);
  L.rec_next = P<unsigned long long>(ctx->rec_next);
  L.out_bytes = P<uint8_t>(ctx->outb);
  L.out_next = P<unsigned long long>(ctx->out_next);
  L.rng_ovl = P<aln::Ovl>(ctx->rng_ovl);
  L.rng_next = P<unsigned long long>(ctx->rng_next);

  return PGA_OK;
}

// Pairs beyond which the alignment launch uses k_align_pairs_wide: 2 x 100 Mbp
// (10 K pairs) is 5 % faster with <2>, 2 x 1 Gbp (101 M pairs) 19 % faster
// with <3>.
constexpr int64_t ALIGN_MANY_PAIRS = 1 << 20;

// Frees what the alignment no longer reads once both diagonal sorts are done
// -- the index (records, LCPs, entries, scratch) and the unsorted seeds -- so
// that a genome too large for all stages' buffers at once still aligns.
// Returns whether anything was freed.
bool release_for_align(pga_ctx *ctx) {
  if (!ctx->have_diag[0] || !ctx->have_diag[1]) return false;
  std::vector<DBuf *> bufs = {&ctx->rec, &ctx->rec2, &ctx->lcp, &ctx->ent, &ctx->seed[0], &ctx->seed[1],
                              &ctx->dlook};
  bool any = false;
  for (DBuf *b : bufs)
    if (b->p) {
      ctx->arena.release(b->p);
      b->p = nullptr;
      b->cap = 0;
      any = true;
    }
  ctx->have_index = ctx->have_entries = false;
  ctx->seeds_released = true;
  return any;
}

// The survivors (ctx->recs, their traces in ctx->outb) in la_sort order into
// ctx->srecs / ctx->strace: keys (fields, then record index) radix-sorted,
// records gathered, trace bytes moved to the scanned offsets.
int la_sort_device(pga_ctx *ctx, int64_t n, int64_t nbytes) {
  ctx->nalign = n;
  ctx->ntrace = nbytes;
  ctx->host_valid = false;
  ENSURE(ctx->srecs, sizeof(AlnRec) * (size_t)n + 16);
  ENSURE(ctx->slen, sizeof(int64_t) * (size_t)(n + 1) + 16);
  ENSURE(ctx->strace, (size_t)nbytes + 16);
  if (n == 0) return PGA_OK;
  const int64_t he = radix_hist_elems(n);
  ENSURE(ctx->skeys, sizeof(U128) * (size_t)n + 16);
  ENSURE(ctx->skeys2, sizeof(U128) * (size_t)n + 16);
  ENSURE(ctx->lhist, sizeof(uint32_t) * (size_t)he + 64);
  ENSURE(ctx->lscan, std::max(sizeof(uint32_t) * (size_t)scan_tmp_elems(he), sizeof(int64_t) * (size_t)scan_tmp_elems(n)) +
                         64);
  ENSURE(ctx->u64tmp, 64);
  U128 *keys = P<U128>(ctx->skeys);
  launch_aln_keys(P<AlnRec>(ctx->recs), n, keys, ctx->st);
  unsigned long long *acc = P<unsigned long long>(ctx->u64tmp);
  CK(cudaMemsetAsync(acc, 0, 16, ctx->st));
  k_u128_diffbits<<<grid_for(n, 256, 148 * 4), 256, 0, ctx->st>>>(keys, n, acc);
  unsigned long long diff[2];
  CK(cudaMemcpyAsync(diff, acc, 16, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  int passes[16], np = 0;
  for (int sh = 0; sh < 128; sh += 8)
    if (((sh < 64 ? diff[0] : diff[1]) >> (sh & 63)) & 0xffull) passes[np++] = sh;
  U128 *res = keys;
  CK(radix_sort_u128(keys, P<U128>(ctx->skeys2), n, passes, np, P<uint32_t>(ctx->lhist), P<uint32_t>(ctx->lscan),
                     &res, ctx->st));
  int64_t *len = P<int64_t>(ctx->slen);
  launch_aln_gather(res, n, P<AlnRec>(ctx->recs), P<AlnRec>(ctx->srecs), len, ctx->st);
  CK(exclusive_scan<int64_t>(len, len, n, P<int64_t>(ctx->lscan), len + n, ctx->st));
  launch_aln_traces(P<AlnRec>(ctx->srecs), len, n, P<uint8_t>(ctx->outb), P<uint8_t>(ctx->strace), ctx->st);
  LAUNCHED(2 + 5 * np + 5);  // keys, bits; np x (hist, 3 scan, scatter); gather, 3 scan, traces
  CK(cudaGetLastError());
  return PGA_OK;
}

// The host copy of the last alignment's results (made on first read).
int host_alignments(pga_ctx *ctx) {
  if (ctx->host_valid) return PGA_OK;
  const int64_t n = ctx->nalign;
  ctx->h_recs.resize(n);
  ctx->h_toff.assign(n + 1, 0);
  ctx->h_trace.clear();
  if (n > 0) {
    CK(cudaMemcpyAsync(ctx->h_recs.data(), ctx->srecs.p, sizeof(AlnRec) * n, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    // the survivors' traces lie back to back from offset 0
    const int64_t total = ctx->h_recs[n - 1].toff + ctx->h_recs[n - 1].tlen;
    if (total < 0 || total > ctx->ntrace) return fail(ctx, PGA_ERR_CUDA, "alignment traces out of range");
    ctx->h_trace.resize(total);
    if (total > 0)
      CK(cudaMemcpyAsync(ctx->h_trace.data(), ctx->strace.p, total, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    for (int64_t i = 0; i < n; i++) ctx->h_toff[i] = ctx->h_recs[i].toff;
    ctx->h_toff[n] = total;
  }
  ctx->host_valid = true;
  return PGA_OK;
}

int run_align(pga_ctx *ctx) {
  const double t_start = now_ms();
  const int nc = ctx->ncontig;
  int64_t maxctg = ctx->maxctg;
  // 1. the two units must be diagonal-sorted
  for (int comp = 0; comp < 2; comp++)
    if (!ctx->have_diag[comp]) {
      int64_t cnt;
      int sw;
      int r = pga_diag_sort(ctx, comp, &sw, &cnt);
      if (r) return r;
    }
  {
    // the aligner's sequences, pools and pair lists need about 16 bytes per
    // input base and 8 per seed beyond the sorted seeds; make room first
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    int64_t seqtot = 0;
    for (int c = 0; c < nc; c++) seqtot += ctx->clen[c];
    const double need = 16.0 * seqtot + 8.0 * (ctx->nseed[0] + ctx->nseed[1]) + (8ll << 30);
    if ((double)free_b + (double)ctx->arena.free_bytes() < need) release_for_align(ctx);
  }
  // 2. NUMERIC and packed sequences, base frequencies, scoring tables
  int ave_path = 0;
  int r0 = prepare_sequences(ctx, &ave_path);
  if (r0) return r0;
  // 3. work spaces (before the pair lists: running out of memory here is
  // cheap to recover from)
  AlignLaunch L{};
  r0 = prepare_workspace(ctx, L, ave_path);
  if (r0) return r0;
  ctx->cand_used = ctx->rng_used = ctx->rec_used = ctx->out_used = 0;
  for (int i = 0; i < 4; i++) ctx->align_work[i] = 0;
  ctx->align_prof[0] = ctx->align_prof[1] = 0;

  // 4. Pair lists of both units.  They stay on the device; only the pairs
  // the host plans come back: self pairs (FastGA's order) and, with band
  // ranges on, pairs of more than RS seeds.  Every other pair becomes a
  // device task, largest first, whose outcome is reduced on the device.
  const int64_t all_seeds = ctx->nseed[0] + ctx->nseed[1];
  // about 160 tasks per warp: short enough that a long alignment's band
  // blocks spread over warps, long enough to keep the per-task cost small
  const int64_t RS = ctx->range_seeds < 0    ? 0
                     : ctx->range_seeds > 0 ? ctx->range_seeds
                                            : std::max<int64_t>(256, all_seeds / (160 * L.nwarps));
  std::vector<PairTask> pairs[2];
  int64_t npairs[2] = {0, 0};
  DBuf *dpst[2] = {&ctx->pstart, &ctx->pstart2}, *dpab[2] = {&ctx->pab, &ctx->pab2};
  // A resident target's Local_Alignment results (requests of the served
  // form): used when the scoring tables are those of the target's run; the
  // target's own run records them (capture)
  const pga_target *rt = ctx->reuse_t;
  for (int i = 0; i < 4; i++) ctx->reuse_stats[i] = 0;
  bool memo_on = false;
  if (rt) {
    const pga_target::Memo &M = rt->memo;
    int why = M.valid ? 0 : 1;
    if (!why && (M.spec != ctx->spec_host || M.ave_path != ctx->ave_path_host)) why = 3;
    ctx->reuse_stats[3] = why;
    if (!why) {
      memo_on = true;
      L.memo.key = P<uint32_t>(M.key);
      L.memo.val = P<int32_t>(M.val);
      L.memo.toff = P<int64_t>(M.toff);
      L.memo.trace = P<uint8_t>(M.trace);
      L.memo.cap = M.cap;
      L.memo.nt = rt->ncontig;
      ENSURE(ctx->memo_hits, 16);
      CK(cudaMemsetAsync(ctx->memo_hits.p, 0, 16, ctx->st));
      L.memo.hits = P<unsigned long long>(ctx->memo_hits);
    }
  }
  if (ctx->capture) {
    const int64_t lc = ctx->cap_calls > 0 ? ctx->cap_calls : 1, lb = ctx->cap_bytes > 0 ? ctx->cap_bytes : 16;
    ENSURE(ctx->mlog_key, sizeof(uint32_t) * MEMO_KEY * (size_t)lc);
    ENSURE(ctx->mlog_val, sizeof(int32_t) * MEMO_VAL * (size_t)lc);
    ENSURE(ctx->mlog_toff, sizeof(int64_t) * (size_t)lc);
    ENSURE(ctx->mlog_trace, (size_t)lb);
    ENSURE(ctx->mlog_ctr, 16);
    CK(cudaMemsetAsync(ctx->mlog_ctr.p, 0, 16, ctx->st));
    L.memo.nt = nc;  // every contig is the target's
    L.memo.lkey = P<uint32_t>(ctx->mlog_key);
    L.memo.lval = P<int32_t>(ctx->mlog_val);
    L.memo.ltoff = P<int64_t>(ctx->mlog_toff);
    L.memo.ltrace = P<uint8_t>(ctx->mlog_trace);
    L.memo.lnext = P<unsigned long long>(ctx->mlog_ctr);
    L.memo.lbytes = L.memo.lnext + 1;
    L.memo.lcap = lc;
    L.memo.lbytes_cap = lb;
  }
  for (int comp = 0; comp < 2; comp++) {
    int64_t n = ctx->nseed[comp];
    if (n == 0) continue;
    ENSURE(ctx->pflag, sizeof(uint32_t) * (n + 1));
    ENSURE(ctx->pidx, sizeof(uint32_t) * (n + 1));
    ENSURE(ctx->scan_tmp, sizeof(uint32_t) * scan_tmp_elems(n + 1) + 64);
    ENSURE(ctx->u64tmp, 64);
    launch_pair_flags(ctx->sorted[comp], n, ctx->lay[comp], P<uint32_t>(ctx->pflag), ctx->st);
    uint32_t *tot = P<uint32_t>(ctx->u64tmp);
    CK(exclusive_scan<uint32_t>(P<uint32_t>(ctx->pflag), P<uint32_t>(ctx->pidx), n, P<uint32_t>(ctx->scan_tmp), tot,
                                ctx->st));
    LAUNCHED(4);
    uint32_t np = 0;
    CK(cudaMemcpyAsync(&np, tot, 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    npairs[comp] = np;
    ENSURE(*dpst[comp], sizeof(int64_t) * (np + 1));
    ENSURE(*dpab[comp], sizeof(int32_t) * 2 * (np + 1));
    const int64_t *pst = P<int64_t>(*dpst[comp]);
    const int32_t *pab = P<int32_t>(*dpab[comp]);
    launch_pair_starts(ctx->sorted[comp], n, ctx->lay[comp], P<uint32_t>(ctx->pflag), P<uint32_t>(ctx->pidx),
                       (int64_t *)pst, (int32_t *)pab, ctx->st);
    // which pairs have a band block that can pass the hit test (the others need no task)
    ENSURE(ctx->plive[comp], (size_t)np + 16);
    CK(cudaMemsetAsync(ctx->plive[comp].p, 0, (size_t)np + 16, ctx->st));
    launch_pair_live(P<uint16_t>(ctx->binfo[comp]), n, P<uint32_t>(ctx->pflag), P<uint32_t>(ctx->pidx),
                     P<uint8_t>(ctx->plive[comp]), ctx->st);
    LAUNCHED(1);
    // the host's pairs
    launch_pair_hostbound(pst, pab, np, n, comp, RS, P<uint32_t>(ctx->pflag), ctx->st);
    CK(exclusive_scan<uint32_t>(P<uint32_t>(ctx->pflag), P<uint32_t>(ctx->pidx), np, P<uint32_t>(ctx->scan_tmp), tot,
                                ctx->st));
    LAUNCHED(5);
    uint32_t nh = 0;
    CK(cudaMemcpyAsync(&nh, tot, 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    std::vector<int64_t> h3(3 * (size_t)nh);
    if (nh > 0) {
      ENSURE(ctx->io2, sizeof(int64_t) * 3 * (size_t)nh);
      launch_pair_gather(pst, pab, np, n, P<uint32_t>(ctx->pflag), P<uint32_t>(ctx->pidx), P<int64_t>(ctx->io2),
                         ctx->st);
      LAUNCHED(1);
      CK(cudaMemcpyAsync(h3.data(), ctx->io2.p, sizeof(int64_t) * 3 * nh, cudaMemcpyDeviceToHost, ctx->st));
      CK(cudaStreamSynchronize(ctx->st));
    }
    for (uint32_t q = 0; q < nh; q++) {
      PairTask t;
      t.comp = comp;
      t.a = (int)(h3[3 * q + 2] >> 32);
      t.b = (int)(uint32_t)h3[3 * q + 2];
      t.self = (comp == 0 && t.a == t.b);
      t.entry_bepos = 0;
      t.seg = -1;
      t.lo = h3[3 * q];
      t.hi = h3[3 * q + 1];
      t.slo = t.lo;
      t.shi = t.hi;
      pairs[comp].push_back(t);
    }
  }
  // the device's pairs: a counting sort by size (largest first) per unit
  int64_t nsmall = 0;
  {
    int64_t cap = 0;
    for (int comp = 0; comp < 2; comp++) cap += npairs[comp] - (int64_t)pairs[comp].size();
    ENSURE(ctx->small, sizeof(uint64_t) * (size_t)(cap + 1));
    ENSURE(ctx->shist, sizeof(uint32_t) * 2 * (SMALL_BINS + 1));
    ENSURE(ctx->scan_tmp, sizeof(uint32_t) * scan_tmp_elems(SMALL_BINS + 1) + 64);
    uint32_t *hist = P<uint32_t>(ctx->shist), *cur = hist + (SMALL_BINS + 1);
    for (int comp = 0; comp < 2; comp++) {
      if (npairs[comp] - (int64_t)pairs[comp].size() <= 0) continue;
      CK(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * (SMALL_BINS + 1), ctx->st));
      launch_small_hist(P<int64_t>(*dpst[comp]), P<int32_t>(*dpab[comp]), npairs[comp], ctx->nseed[comp], comp, RS,
                        P<uint8_t>(ctx->plive[comp]), hist, ctx->st);
      uint32_t *tot = P<uint32_t>(ctx->u64tmp);
      CK(exclusive_scan<uint32_t>(hist, cur, SMALL_BINS + 1, P<uint32_t>(ctx->scan_tmp), tot, ctx->st));
      uint32_t ns = 0;
      CK(cudaMemcpyAsync(&ns, tot, 4, cudaMemcpyDeviceToHost, ctx->st));
      launch_small_scatter(P<int64_t>(*dpst[comp]), P<int32_t>(*dpab[comp]), npairs[comp], ctx->nseed[comp], comp, RS,
                           P<uint8_t>(ctx->plive[comp]), cur, P<uint64_t>(ctx->small) + nsmall, ctx->st);
      CK(cudaStreamSynchronize(ctx->st));
      LAUNCHED(5);
      nsmall += ns;
    }
    CK(cudaGetLastError());
  }
  if (nsmall >= (int64_t)0x7fffffff - 16)
    return fail(ctx, PGA_ERR_LIMIT, "%lld contig pairs: at most 2^31 supported", (long long)nsmall);
  // FastGA's order of the contigs (GIXmake's: longest first, stable)
  FastgaOrder F;
  F.n = nc;
  F.at.resize(nc);
  for (int i = 0; i < nc; i++) F.at[i] = i;
  std::stable_sort(F.at.begin(), F.at.end(), [&](int x, int y) { return ctx->clen[x] > ctx->clen[y]; });
  F.pos.resize(nc);
  for (int i = 0; i < nc; i++) F.pos[F.at[i]] = i;
  ENSURE(ctx->fo_dev, sizeof(int) * (size_t)nc + sizeof(unsigned long long) * (8 + 2 * (size_t)nc) + 16);
  int *fo_pos = P<int>(ctx->fo_dev);
  unsigned long long *sred = (unsigned long long *)(P<uint8_t>(ctx->fo_dev) + ((sizeof(int) * (size_t)nc + 15) & ~15));
  CK(cudaMemcpyAsync(fo_pos, F.pos.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, ctx->st));
  L.small = P<uint64_t>(ctx->small);
  L.nsmall = (int)nsmall;
  for (int u = 0; u < 2; u++) {
    L.pstart[u] = P<int64_t>(*dpst[u]);
    L.pab[u] = P<int32_t>(*dpab[u]);
    L.npairs[u] = npairs[u];
    L.nseeds[u] = ctx->nseed[u];
  }
  L.fo_pos = fo_pos;
  // the launch is bounded by its longest tasks up to about a million pairs,
  // by throughput beyond: then the build with more resident warps
  L.min_blocks = ctx->align_build ? ctx->align_build : npairs[0] + npairs[1] > ALIGN_MANY_PAIRS ? 5 : 2;
  L.sred = sred;
  L.fo_last = sred + 8;
  L.fo_earlier = sred + 8 + nc;

  // 5. Plan.  Pairs of two different contigs (all C pairs, every N pair of
  // two contigs) run in the first launch, large ones as band ranges finished
  // right after.  A self pair reads what the previous pair left in `path`
  // only in a chain that straddles diagonal 0, i.e. only in its band blocks
  // whose diagonal span holds 0 (bands cd_lo..cd_hi); its blocks below and
  // above that run as ranges in the first launch too, and its middle part
  // runs in rounds of FastGA's order, entered with the bepos of the last call
  // below it (or, if none, the order's value).  With ranges off, self pairs
  // run whole in the rounds.
  std::vector<PairTask> first;
  std::vector<int> self_idx;
  for (int comp = 0; comp < 2; comp++)
    for (size_t i = 0; i < pairs[comp].size(); i++) {
      if (pairs[comp][i].self) self_idx.push_back((int)i);
      else first.push_back(pairs[comp][i]);
    }
  const int nself = (int)self_idx.size();
  std::vector<int64_t> x12(2 * (size_t)nself, 0);
  if (RS > 0 && nself > 0) {
    const int64_t bmx = maxctg, num = bmx - 127;
    const int64_t cd_lo = num >= 0 ? (num + 63) / 64 : -((-num) / 64), cd_hi = bmx / 64;
    std::vector<int64_t> lohi(2 * (size_t)nself);
    for (int q = 0; q < nself; q++) {
      lohi[2 * q] = pairs[0][self_idx[q]].lo;
      lohi[2 * q + 1] = pairs[0][self_idx[q]].hi;
    }
    ENSURE(ctx->selfb, sizeof(int64_t) * 4 * (size_t)nself);
    int64_t *dlohi = P<int64_t>(ctx->selfb), *dx12 = dlohi + 2 * nself;
    CK(cudaMemcpyAsync(dlohi, lohi.data(), sizeof(int64_t) * 2 * nself, cudaMemcpyHostToDevice, ctx->st));
    launch_self_bounds(ctx->sorted[0], ctx->lay[0], dlohi, nself, cd_lo, cd_hi, dx12, ctx->st);
    LAUNCHED(1);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(x12.data(), dx12, sizeof(int64_t) * 2 * nself, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
  int nranges = 0;
  // ranges of about RS seeds covering seeds [x0, x1) of pair t (x1 a band start)
  auto add_ranges = [&](const PairTask &t, int64_t x0, int64_t x1, std::vector<int> &ids,
                        std::vector<PairTask> &dst) {
    const int64_t step = RS > 0 ? RS : x1 - x0;
    for (int64_t x = x0; x < x1; x += step) {
      PairTask r = t;
      r.entry_bepos = 0;
      r.seg = nranges++;
      r.slo = x;
      r.shi = std::min(x1, x + step);
      ids.push_back(r.seg);
      dst.push_back(r);
    }
  };
  LaunchPlan P1;
  std::vector<int> first_task(first.size(), -1), first_fin(first.size(), -1);
  std::vector<std::vector<int>> first_ids(first.size());
  struct SelfPlan {
    std::vector<int> pre, post;
    int diag = -1;  // range number of the middle part (RS > 0)
    bool whole = false;
  };
  std::vector<SelfPlan> sp(nself);
  std::vector<PairTask> diag_task(nself);
  // The launch's tasks, largest pair first (a large pair's ranges each tend
  // to re-extend its longest alignments, so they start early): pairs of two
  // contigs (id >= 0) and the outer parts of self pairs (id = -1 - q).
  std::vector<std::pair<int64_t, int>> src;
  for (size_t i = 0; i < first.size(); i++) src.push_back({first[i].hi - first[i].lo, (int)i});
  if (RS > 0)
    for (int q = 0; q < nself; q++) {
      const PairTask &t = pairs[0][self_idx[q]];
      src.push_back({t.hi - t.lo, -1 - q});
    }
  std::stable_sort(src.begin(), src.end(), [](const std::pair<int64_t, int> &x, const std::pair<int64_t, int> &y) {
    return x.first > y.first;
  });
  {
    size_t est = 2 * (size_t)nself + 1;
    for (const auto &s : src) est += RS > 0 ? (size_t)(s.first / RS + 2) : 1;
    P1.tasks.reserve(est);
    P1.ridx.reserve(est);
  }
  for (const auto &s : src) {
    if (s.second >= 0) {
      const size_t i = (size_t)s.second;
      PairTask t = first[i];
      if (RS > 0 && t.hi - t.lo > RS) {
        add_ranges(t, t.lo, t.hi, first_ids[i], P1.tasks);
        FinishTask f{t.comp, t.a, t.b, 0, (int)P1.ridx.size(), (int)first_ids[i].size()};
        P1.ridx.insert(P1.ridx.end(), first_ids[i].begin(), first_ids[i].end());
        first_fin[i] = (int)P1.fins.size();
        P1.fins.push_back(f);
      } else {
        first_task[i] = (int)P1.tasks.size();
        P1.tasks.push_back(t);
      }
    } else {
      const int q = -1 - s.second;
      const PairTask &t = pairs[0][self_idx[q]];
      const int64_t x1 = t.lo + x12[2 * q], x2 = t.lo + x12[2 * q + 1];
      add_ranges(t, t.lo, x1, sp[q].pre, P1.tasks);
      add_ranges(t, x2, t.hi, sp[q].post, P1.tasks);
    }
  }
  for (int q = 0; q < nself; q++) {
    const PairTask &t = pairs[0][self_idx[q]];
    if (RS <= 0) {
      sp[q].whole = true;
      diag_task[q] = t;
      continue;
    }
    const int64_t x1 = t.lo + x12[2 * q], x2 = t.lo + x12[2 * q + 1];
    if (x2 > x1) {
      PairTask d = t;
      d.seg = sp[q].diag = nranges++;
      d.slo = x1;
      d.shi = x2;
      diag_task[q] = d;
    }
  }
  ENSURE(ctx->rout, sizeof(PairOut) * (size_t)(nranges + 1));
  std::vector<PairOut> rout_h(nranges);

  const double t_launch = now_ms();
  long long maxcyc = 0, sumcyc = 0;
  int64_t maxcalls = 0, calls = 0;
  std::vector<PairOut> tout, fout;
  int r = align_launch(ctx, L, P1, tout, fout, rout_h, &maxcyc, &maxcalls);
  if (r) return r;
  // the device-planned pairs: totals and, per order position, FastGA's
  // order keys of the N pairs among them
  std::vector<int64_t> Lk(nc, 0), ebest(nc, 0);
  if (L.nsmall > 0) {
    unsigned long long red[8];
    std::vector<unsigned long long> fo(2 * (size_t)nc);
    CK(cudaMemcpyAsync(red, L.sred, sizeof(red), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(fo.data(), L.fo_last, sizeof(unsigned long long) * 2 * nc, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    calls += (int64_t)red[0];
    sumcyc += (long long)red[1];
    for (int x = 0; x < nc; x++) {
      Lk[x] = (int64_t)fo[x];
      ebest[x] = (int64_t)fo[nc + x];
    }
  }
  L.nsmall = 0;  // the later launches run host-planned tasks only
  std::vector<PairOut> out1(first.size());
  for (size_t i = 0; i < first.size(); i++) {
    if (first_task[i] >= 0) {
      out1[i] = tout[first_task[i]];
    } else {
      out1[i] = fout[first_fin[i]];
      long long c = 0;
      for (int id : first_ids[i]) c += rout_h[id].cycles;
      out1[i].cycles = c + fout[first_fin[i]].cycles;
    }
    calls += out1[i].calls;
    sumcyc += out1[i].cycles;
  }

  const double t_self = now_ms();
  // 6. self pairs: entry values by FastGA's order (src/fastga_order.c)
  int64_t nrounds = 0;
  if (nself > 0) {
    // seeds of each anchor contig in the N unit (its diagonal-sort panel)
    std::vector<int64_t> panel(nc + 1, 0), nseeds(nc, 0);
    ENSURE(ctx->panel[0], sizeof(int64_t) * (nc + 1));
    k_panel_bounds<<<(nc + 1 + 255) / 256, 256, 0, ctx->st>>>(ctx->sorted[0], ctx->nseed[0], ctx->lay[0], nc,
                                                             P<int64_t>(ctx->panel[0]));
    LAUNCHED(1);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(panel.data(), ctx->panel[0].p, sizeof(int64_t) * (nc + 1), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    for (int c = 0; c < nc; c++) nseeds[c] = panel[c + 1] - panel[c];
    std::vector<int64_t> clen_pos(nc), seeds_pos(nc);
    int64_t seqtot = 0;
    for (int i = 0; i < nc; i++) {
      clen_pos[i] = ctx->clen[F.at[i]];
      seeds_pos[i] = nseeds[F.at[i]];
      seqtot += ctx->clen[i];
    }
    int swide = 2 * ctx->lay[0].dbyte + ctx->ctgb + 2;
    fo_ranges(nc, clen_pos, seqtot, seeds_pos, swide, 32, F.range_start);
    // results of the N pairs of two contigs, by anchor position: the
    // largest key of a pair that called (Lk) and of one whose partner comes
    // earlier in the order (ebest: the nearest earlier partner that called);
    // the device-planned pairs' share came from their reduction
    for (size_t i = 0; i < first.size(); i++) {
      const PairTask &t = first[i];
      if (t.comp || out1[i].calls <= 0) continue;
      int xa = F.pos[t.a], xb = F.pos[t.b];
      int64_t key = fo_key(xb, out1[i].exit_bepos);
      if (key > Lk[xa]) Lk[xa] = key;
      if (xb < xa && key > ebest[xa]) ebest[xa] = key;
    }
    const int UNSET_MAIN = 32767;
    auto unset = [&](int rs) { return rs == 0 ? UNSET_MAIN : 0; };
    std::vector<int64_t> S(nc, 0);  // 0 none, 1 pending, 2 no call, 3+bepos called
    std::vector<int> val(nself, 0), state(nself, 0);  // 0 undetermined, 1 known
    std::vector<char> done(nself, 0);
    // the ranges of self pair q in order, with its middle part's
    auto self_ids = [&](int q) {
      std::vector<int> ids = sp[q].pre;
      if (sp[q].diag >= 0) ids.push_back(sp[q].diag);
      ids.insert(ids.end(), sp[q].post.begin(), sp[q].post.end());
      return ids;
    };
    LaunchPlan pending;  // self pairs to finish in the next launch
    std::vector<int> pending_q;
    for (int q = 0; q < nself; q++) {
      const PairTask &t = pairs[0][self_idx[q]];
      int x = F.pos[t.a];
      S[x] = 1;
      if (!sp[q].whole) {
        int pc, pe;
        combine_ranges(rout_h, sp[q].pre, &pc, &pe, 0);
        if (pc > 0 || sp[q].diag < 0) {
          // entered after a call of its own, or with no middle part: its
          // result does not depend on the order's value
          val[q] = pe;
          state[q] = 1;
          if (sp[q].diag < 0) {
            std::vector<int> ids = self_ids(q);
            int c, e;
            combine_ranges(rout_h, ids, &c, &e, 0);
            S[x] = c > 0 ? 3 + (int64_t)e : 2;
            calls += c;
            for (int id : ids) sumcyc += rout_h[id].cycles;
            done[q] = 1;
            FinishTask f{0, t.a, t.b, 0, (int)pending.ridx.size(), (int)ids.size()};
            pending.ridx.insert(pending.ridx.end(), ids.begin(), ids.end());
            pending.fins.push_back(f);
          }
          continue;
        }
      }
      // nearest earlier partner that made a call (src/fastga_order_core.c:147-166)
      const bool found = ebest[x] != 0;
      if (found) val[q] = (int)(ebest[x] & 0xffffffffll);
      if (found) state[q] = 1;
      else if (F.range_start[x] == x) {
        val[q] = unset(F.range_start[x]);
        state[q] = 1;
      }
    }
    while (true) {
      LaunchPlan plan = pending;
      pending = LaunchPlan();
      std::vector<int> bq;
      for (int q = 0; q < nself; q++) {
        if (done[q]) continue;
        if (!state[q]) {
          // fo_from_rows (src/fastga_order_core.c:167-192)
          const PairTask &t = pairs[0][self_idx[q]];
          int x = F.pos[t.a], rs = F.range_start[x];
          bool known = false, wait = false;
          int bep = 0;
          for (int y = x - 1; y >= rs; y--) {
            int64_t k = Lk[y], sv = S[y];
            if (k != 0 && (int)(k >> 32) - 1 > y) {
              bep = (int)(k & 0xffffffffll);
              known = true;
            } else if (sv == 1) {
              wait = true;
            } else if (sv >= 3) {
              bep = (int)(sv - 3);
              known = true;
            } else if (k != 0) {
              bep = (int)(k & 0xffffffffll);
              known = true;
            } else
              continue;
            break;
          }
          if (wait) continue;
          val[q] = known ? bep : unset(rs);
          state[q] = 1;
        }
        PairTask d = diag_task[q];
        d.entry_bepos = val[q];
        plan.tasks.push_back(d);
        bq.push_back(q);
        if (!sp[q].whole) {
          std::vector<int> ids = self_ids(q);
          FinishTask f{0, d.a, d.b, 0, (int)plan.ridx.size(), (int)ids.size()};
          plan.ridx.insert(plan.ridx.end(), ids.begin(), ids.end());
          plan.fins.push_back(f);
        }
      }
      if (plan.tasks.empty() && plan.fins.empty()) break;
      if (!plan.tasks.empty()) nrounds++;
      r = align_launch(ctx, L, plan, tout, fout, rout_h, &maxcyc, &maxcalls);
      if (r) return r;
      for (size_t i = 0; i < bq.size(); i++) {
        const int q = bq[i];
        done[q] = 1;
        int x = F.pos[pairs[0][self_idx[q]].a];
        int c, e;
        if (sp[q].whole) {
          c = tout[i].calls;
          e = tout[i].exit_bepos;
          sumcyc += tout[i].cycles;
        } else {
          std::vector<int> ids = self_ids(q);
          combine_ranges(rout_h, ids, &c, &e, val[q]);
          for (int id : ids) sumcyc += rout_h[id].cycles;
        }
        S[x] = c > 0 ? 3 + (int64_t)e : 2;
        calls += c;
      }
    }
    for (int q = 0; q < nself; q++)
      if (!done[q]) return fail(ctx, PGA_ERR_ARG, "self pairs that cannot be resolved");
  }

  const double t_order = now_ms();
  // 7. survivors in la_sort order: (aread, abpos, bread, comp), ties in the
  // pair's own output order (src/fastga_pipeline.c:1500-1515), on the device
  if (memo_on) {
    unsigned long long hits = 0;
    CK(cudaMemcpyAsync(&hits, ctx->memo_hits.p, 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->reuse_stats[0] = 1;
    ctx->reuse_stats[1] = (int64_t)hits;
    ctx->reuse_stats[2] = calls;
  }
  unsigned long long nrec = 0, nbytes = 0;
  CK(cudaMemcpyAsync(&nrec, ctx->rec_next.p, 8, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaMemcpyAsync(&nbytes, ctx->out_next.p, 8, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  r0 = la_sort_device(ctx, (int64_t)nrec, (int64_t)nbytes);
  if (r0) return r0;
  ctx->align_stats[0] = npairs[0] + npairs[1];
  ctx->align_stats[1] = (int64_t)self_idx.size();
  ctx->align_stats[2] = calls;
  ctx->align_stats[3] = maxcyc;
  ctx->align_stats[4] = (int64_t)nrec;
  ctx->align_stats[5] = nrounds;
  ctx->align_stats[6] = sumcyc;
  ctx->align_stats[7] = maxcalls;
  ctx->align_work[2] = calls;
  const double t_end = now_ms();
  ctx->align_ms[0] = (float)(t_launch - t_start);
  ctx->align_ms[1] = (float)(t_self - t_launch);
  ctx->align_ms[2] = (float)(t_order - t_self);
  ctx->align_ms[3] = (float)(t_end - t_order);
  ctx->have_align = true;
  return PGA_OK;
}
}  // namespace

// =============================================================================
// C ABI
// =============================================================================

extern "C" {

int pga_ctx_create(int device, pga_ctx **out) {
  if (!out) return PGA_ERR_ARG;
  *out = nullptr;
  pga_ctx *ctx = new (std::nothrow) pga_ctx();
  if (!ctx) return PGA_ERR_NOMEM;
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete ctx;
    return PGA_ERR_CUDA;
  }
  ctx->st = ctx->own;
  for (int s = 0; s < ST_N; s++) {
    cudaEventCreate(&ctx->ev[s][0]);
    cudaEventCreate(&ctx->ev[s][1]);
  }
  *out = ctx;
  return PGA_OK;
}

void pga_ctx_destroy(pga_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->st);
  DBuf *abufs[] = {&ctx->pk, &ctx->poff, &ctx->pwords, &ctx->numf, &ctx->numr, &ctx->soff, &ctx->spec_tab, &ctx->tasks, &ctx->task_next, &ctx->pout, &ctx->binfo[0], &ctx->binfo[1], &ctx->plive[0], &ctx->plive[1],
                   &ctx->wave, &ctx->points, &ctx->cells, &ctx->cell_next, &ctx->ovl, &ctx->perm, &ctx->cand,
                   &ctx->cand_next, &ctx->recs, &ctx->rec_next, &ctx->outb, &ctx->out_next, &ctx->pflag,
                   &ctx->pidx, &ctx->pstart, &ctx->pab, &ctx->rng_ovl, &ctx->rng_next, &ctx->ftasks,
                   &ctx->fout, &ctx->ridx, &ctx->rout, &ctx->selfb, &ctx->lreq, &ctx->lpath, &ctx->ltoff,
                   &ctx->ltrace, &ctx->lnext, &ctx->pstart2, &ctx->pab2, &ctx->small, &ctx->shist, &ctx->fo_dev,
                   &ctx->srecs, &ctx->slen, &ctx->strace, &ctx->skeys, &ctx->skeys2, &ctx->lhist, &ctx->lscan,
                   &ctx->memo_hits, &ctx->mlog_key, &ctx->mlog_val, &ctx->mlog_toff, &ctx->mlog_trace,
                   &ctx->mlog_ctr};
  for (DBuf *b : abufs) ctx->arena.release(b->p);
  DBuf *bufs[] = {&ctx->bps, &ctx->dclen, &ctx->dboff, &ctx->tile_ctg, &ctx->tile_j0, &ctx->hist, &ctx->start,
                  &ctx->scan_tmp, &ctx->rec, &ctx->rec2, &ctx->lcp, &ctx->ent, &ctx->cum, &ctx->qmed,
                  &ctx->qbig, &ctx->qcount, &ctx->maxrun, &ctx->u64tmp, &ctx->blk_n, &ctx->blk_c,
                  &ctx->blk_tmp, &ctx->seed[0], &ctx->seed[1], &ctx->keys[0], &ctx->keys[1],
                  &ctx->dlook, &ctx->dsmall, &ctx->panel[0], &ctx->panel[1], &ctx->io,
                  &ctx->io2, &ctx->coarse, &ctx->fa_text, &ctx->fa_mask, &ctx->fa_seq, &ctx->fa_cnt, &ctx->fa_tmp,
                  &ctx->fa_tot, &ctx->fa_status, &ctx->fa_hdr, &ctx->fa_hbytes, &ctx->fa_runs, &ctx->fa_ctg};
  for (DBuf *b : bufs) ctx->arena.release(b->p);
  ctx->arena.clear();
  for (int s = 0; s < ST_N; s++) {
    cudaEventDestroy(ctx->ev[s][0]);
    cudaEventDestroy(ctx->ev[s][1]);
  }
  for (cudaEvent_t e : ctx->fa_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->own) cudaStreamDestroy(ctx->own);
  delete ctx;
}

const char *pga_last_error(const pga_ctx *ctx) { return ctx ? ctx->err : "null context"; }

int pga_ctx_set_stream(pga_ctx *ctx, void *stream) {
  if (!ctx) return PGA_ERR_ARG;
  // the arena reuses freed ranges in stream order: drain the old stream
  CK(cudaStreamSynchronize(ctx->st));
  ctx->st = stream ? (cudaStream_t)stream : ctx->own;
  return PGA_OK;
}

int pga_ctx_synchronize(pga_ctx *ctx) {
  if (!ctx) return PGA_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->st));
  return PGA_OK;
}

int64_t pga_kernel_launches(const pga_ctx *ctx) { return ctx ? ctx->launches : 0; }

int pga_ctx_enable_timing(pga_ctx *ctx, int on) {
  if (!ctx) return PGA_ERR_ARG;
  ctx->timing = on != 0;
  for (int s = 0; s < ST_N; s++) ctx->stage_used[s] = false;
  for (int s = 0; s <= ST_N; s++) ctx->alloc_ms[s] = 0;
  ctx->alloc_calls = 0;
  return PGA_OK;
}

int pga_alloc_times(const pga_ctx *ctx, double *ms11, int64_t *counts4) {
  if (!ctx || !ms11) return PGA_ERR_ARG;
  for (int s = 0; s <= ST_N; s++) ms11[s] = ctx->alloc_ms[s];
  if (counts4) {
    counts4[0] = ctx->alloc_calls;
    counts4[1] = (int64_t)ctx->arena.held_bytes();
    counts4[2] = (int64_t)ctx->arena.free_bytes();
    counts4[3] = ctx->sheds;
  }
  return PGA_OK;
}

int pga_stage_times(const pga_ctx *cctx, float *ms10) {
  pga_ctx *ctx = const_cast<pga_ctx *>(cctx);
  if (!ctx || !ms10) return PGA_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->st));
  for (int s = 0; s < ST_N; s++) {
    ms10[s] = 0.f;
    if (ctx->stage_used[s]) cudaEventElapsedTime(&ms10[s], ctx->ev[s][0], ctx->ev[s][1]);
  }
  return PGA_OK;
}

namespace {

// Contig table of a GDB whose sequence image is already on the device:
// validation, record sizing and the extraction tiles.
int gdb_tables(pga_ctx *ctx, int ncontig, const int64_t *clen, const int64_t *boff, int64_t bps_bytes) {
  ctx->ncontig = ncontig;
  ctx->bps_bytes = bps_bytes;
  ctx->clen.assign(clen, clen + ncontig);
  ctx->boff.assign(boff, boff + ncontig);
  ctx->maxctg = 0;
  for (int i = 0; i < ncontig; i++) {
    if (clen[i] < 0) return fail(ctx, PGA_ERR_ARG, "contig %d has negative length", i);
    if (clen[i] >= ((int64_t)1 << 31)) return fail(ctx, PGA_ERR_LIMIT, "contig %d longer than 2^31-1", i);
    if (boff[i] >= 0 && boff[i] + (clen[i] + 3) / 4 > bps_bytes)
      return fail(ctx, PGA_ERR_ARG, "contig %d extends past the sequence image", i);
    ctx->maxctg = std::max(ctx->maxctg, clen[i]);
  }
  ctx->posb = bytes_inclusive(ctx->maxctg);
  ctx->ctgb = bytes_inclusive(2 * (int64_t)ncontig - 1);
  if (ctx->ctgb < 1) ctx->ctgb = 1;
  ctx->rsize = 12 + ctx->posb + ctx->ctgb;
  std::vector<int64_t> tj;
  ctx->h_tile_ctg.clear();
  for (int r = 0; r < ncontig; r++) {
    if (boff[r] < 0 || clen[r] < TMER) continue;
    int64_t npos = clen[r] - TMER + 1;
    for (int64_t j0 = 0; j0 < npos; j0 += EXT_TILE) {
      ctx->h_tile_ctg.push_back(r);
      tj.push_back(j0);
    }
  }
  ctx->ntiles = (int)tj.size();
  ENSURE(ctx->tile_ctg, sizeof(int32_t) * (ctx->ntiles + 1));
  ENSURE(ctx->tile_j0, sizeof(int64_t) * (ctx->ntiles + 1));
  if (ctx->ntiles > 0) {
    CK(cudaMemcpyAsync(ctx->tile_ctg.p, ctx->h_tile_ctg.data(), sizeof(int32_t) * ctx->ntiles,
                       cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->tile_j0.p, tj.data(), sizeof(int64_t) * ctx->ntiles, cudaMemcpyHostToDevice, ctx->st));
  }
  CK(cudaStreamSynchronize(ctx->st));
  return PGA_OK;
}

// A new GDB invalidates everything computed from the previous one.
void gdb_reset(pga_ctx *ctx) {
  ctx->have_gdb = false;
  ctx->have_scaffolds = false;
  ctx->freq_set = false;
  ctx->have_index = false;
  ctx->have_seeds = false;
  ctx->have_numeric = false;
  ctx->have_diag[0] = ctx->have_diag[1] = false;
  ctx->have_align = false;
  ctx->reuse_t = nullptr;
}

}  // namespace

int pga_gdb_load(pga_ctx *ctx, const uint8_t *bps, int64_t bps_bytes, int ncontig, const int64_t *clen,
                 const int64_t *boff) {
  if (!ctx || ncontig < 0 || (ncontig > 0 && (!clen || !boff)) || bps_bytes < 0) return PGA_ERR_ARG;
  if (ncontig >= 32768) return fail(ctx, PGA_ERR_LIMIT, "%d contigs: at most 32767 supported", ncontig);
  CK(cudaSetDevice(ctx->device));
  gdb_reset(ctx);
  ENSURE(ctx->bps, (size_t)bps_bytes + 16);
  ENSURE(ctx->dclen, sizeof(int64_t) * (ncontig + 1));
  ENSURE(ctx->dboff, sizeof(int64_t) * (ncontig + 1));
  if (bps_bytes > 0) CK(cudaMemcpyAsync(ctx->bps.p, bps, bps_bytes, cudaMemcpyHostToDevice, ctx->st));
  if (ncontig > 0) {
    CK(cudaMemcpyAsync(ctx->dclen.p, clen, sizeof(int64_t) * ncontig, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->dboff.p, boff, sizeof(int64_t) * ncontig, cudaMemcpyHostToDevice, ctx->st));
  }
  int r = gdb_tables(ctx, ncontig, clen, boff, bps_bytes);
  if (r != PGA_OK) return r;
  ctx->have_gdb = true;
  return PGA_OK;
}

namespace {

// Queues a copy of `count` values of `size` bytes at device address `src`
// into `dst` (stream order).
int fetch_n(pga_ctx *ctx, void *dst, const void *src, int64_t count, size_t size) {
  if (count <= 0) return PGA_OK;
  CK(cudaMemcpyAsync(dst, src, size * count, cudaMemcpyDeviceToHost, ctx->st));
  return PGA_OK;
}
#define fetch(ctx, dst, src, count) fetch_n((ctx), (dst), (src), (count), sizeof(*(dst)))

#define TRY(x)                  \
  do {                          \
    int _r = (x);               \
    if (_r != PGA_OK) return _r; \
  } while (0)

// The device half of pga_gdb_ingest_fasta: text already in ctx->fa_text.
int ingest_device(pga_ctx *ctx, int64_t n, int nthr, int64_t *sizes6) {
  cudaStream_t st = ctx->st;
  const int64_t nt = (n + FA_TILE - 1) / FA_TILE;
  unsigned long long *status;
  int64_t *tot;
  ENSURE(ctx->fa_status, sizeof(unsigned long long) * (FA_NSTATUS + 256));
  ENSURE(ctx->fa_tot, sizeof(int64_t) * 8);
  ENSURE(ctx->fa_cnt, sizeof(int64_t) * 2 * (nt + 1));
  ENSURE(ctx->fa_tmp, sizeof(int64_t) * scan_tmp_elems(nt));
  status = P<unsigned long long>(ctx->fa_status);
  tot = P<int64_t>(ctx->fa_tot);
  int64_t *cnt = P<int64_t>(ctx->fa_cnt), *cnt2 = cnt + (nt + 1);
  const uint8_t *text = P<uint8_t>(ctx->fa_text);
  int64_t h[8];
  unsigned long long hs[FA_NSTATUS + 256];

  // headers
  CK(fa_init_status(status, st));
  CK(fa_count_headers(text, n, cnt, status, st));
  CK(exclusive_scan<int64_t>(cnt, cnt, nt, P<int64_t>(ctx->fa_tmp), tot + 0, st));
  LAUNCHED(5);
  TRY(fetch(ctx, h, tot, 1));
  TRY(fetch(ctx, hs, status, FA_NSTATUS));
  CK(cudaStreamSynchronize(st));
  if (hs[FA_BAD] != ~0ull)
    return fail(ctx, PGA_ERR_ARG, "byte %llu of the text is NUL or not ASCII", hs[FA_BAD]);
  const int64_t nh64 = h[0];
  if (nh64 >= 32768) return fail(ctx, PGA_ERR_LIMIT, "%lld scaffolds: at most 32767 supported", (long long)nh64);
  const int nh = (int)nh64;
  // per scaffold: hstart hend htext hlen1 hoff sstart(+1) trail scf4(4)
  ENSURE(ctx->fa_hdr, sizeof(int64_t) * 11 * (nh + 1));
  int64_t *hstart = P<int64_t>(ctx->fa_hdr), *hend = hstart + (nh + 1), *htext = hend + (nh + 1),
          *hlen1 = htext + (nh + 1), *hoff = hlen1 + (nh + 1), *sstart = hoff + (nh + 1),
          *trail = sstart + (nh + 1), *scf4 = trail + (nh + 1);
  ENSURE(ctx->fa_mask, sizeof(uint32_t) * ((n + 31) / 32 + 4));
  uint32_t *mask = P<uint32_t>(ctx->fa_mask);
  CK(fa_write_headers(text, n, cnt, hstart, st));
  CK(fa_header_lines(text, hstart, nh, hend, htext, hlen1, st));
  ENSURE(ctx->fa_tmp, sizeof(int64_t) * std::max(scan_tmp_elems(nt), scan_tmp_elems(nh)));
  CK(exclusive_scan<int64_t>(hlen1, hoff, nh, P<int64_t>(ctx->fa_tmp), tot + 1, st));
  CK(cudaMemsetAsync(mask, 0, sizeof(uint32_t) * ((n + 31) / 32 + 4), st));
  CK(fa_paint_headers(hstart, hend, nh, mask, st));
  // sequence characters; their total is sstart[nh]
  CK(fa_count_seq(text, n, mask, cnt, st));
  CK(exclusive_scan<int64_t>(cnt, cnt, nt, P<int64_t>(ctx->fa_tmp), sstart + nh, st));
  CK(cudaMemsetAsync(trail, 0, sizeof(int64_t) * (nh + 1), st));
  LAUNCHED(10);
  TRY(fetch(ctx, h + 1, tot + 1, 1));
  TRY(fetch(ctx, h + 2, sstart + nh, 1));
  CK(cudaStreamSynchronize(st));
  const int64_t hdrtot = h[1], G = h[2];
  if (G == 0) return fail(ctx, PGA_ERR_ARG, "missing sequence entry for scaffold 0");
  ENSURE(ctx->fa_hbytes, (size_t)hdrtot + 16);
  ENSURE(ctx->fa_seq, (size_t)G + 64);
  uint8_t *seq = P<uint8_t>(ctx->fa_seq);
  CK(fa_copy_headers(text, htext, hlen1, hoff, nh, P<char>(ctx->fa_hbytes), st));
  CK(cudaMemsetAsync(seq + G, 0, 64, st));
  CK(fa_write_seq(text, n, mask, cnt, hend, nh, seq, sstart, status, st));
  CK(fa_flag_scaffolds(seq, sstart, nh, status, st));
  // N runs
  const int64_t gt = (G + FA_TILE - 1) / FA_TILE;
  ENSURE(ctx->fa_cnt, sizeof(int64_t) * 2 * (std::max(nt, gt) + 1));
  cnt = P<int64_t>(ctx->fa_cnt);
  cnt2 = cnt + (gt + 1);
  ENSURE(ctx->fa_tmp, sizeof(int64_t) * std::max(scan_tmp_elems(gt), scan_tmp_elems(nh)));
  CK(fa_count_runs(seq, G, cnt, cnt2, st));
  CK(exclusive_scan<int64_t>(cnt, cnt, gt, P<int64_t>(ctx->fa_tmp), tot + 2, st));
  CK(exclusive_scan<int64_t>(cnt2, cnt2, gt, P<int64_t>(ctx->fa_tmp), tot + 3, st));
  LAUNCHED(10);
  TRY(fetch(ctx, h + 3, tot + 2, 2));
  TRY(fetch(ctx, hs, status, FA_NSTATUS));
  CK(cudaStreamSynchronize(st));
  if (hs[FA_EMPTY] != ~0ull)
    return fail(ctx, PGA_ERR_ARG, "missing sequence entry for scaffold %llu", hs[FA_EMPTY]);
  const int64_t R = h[3];
  if (h[4] != R) return fail(ctx, PGA_ERR_CUDA, "ingest: %lld run starts but %lld run ends", (long long)R,
                              (long long)h[4]);
  // per run: rs re is_split sr ; rscaf (int32)
  ENSURE(ctx->fa_runs, sizeof(int64_t) * 4 * (R + 1) + sizeof(int32_t) * (R + 1));
  int64_t *rs = P<int64_t>(ctx->fa_runs), *re = rs + (R + 1), *isp = re + (R + 1), *sr = isp + (R + 1);
  int32_t *rscaf = (int32_t *)(sr + (R + 1));
  ENSURE(ctx->fa_tmp, sizeof(int64_t) * std::max(scan_tmp_elems(R), scan_tmp_elems(nh)));
  if (R > 0) {
    CK(fa_write_runs(seq, G, cnt, cnt2, rs, re, st));
    CK(fa_classify_runs(rs, re, R, sstart, nh, nthr, isp, rscaf, trail, status, st));
    LAUNCHED(5);
  }
  CK(exclusive_scan<int64_t>(isp, sr, R, P<int64_t>(ctx->fa_tmp), tot + 4, st));
  TRY(fetch(ctx, h + 5, tot + 4, 1));
  TRY(fetch(ctx, hs, status, FA_NSTATUS));
  CK(cudaStreamSynchronize(st));
  if (hs[FA_ALLN] != ~0ull)
    return fail(ctx, PGA_ERR_ARG, "missing sequence entry for scaffold %llu (all N)", hs[FA_ALLN]);
  const int64_t nsplit = h[5], nc64 = nh + nsplit;
  if (nc64 >= 32768) return fail(ctx, PGA_ERR_LIMIT, "%lld contigs: at most 32767 supported", (long long)nc64);
  const int nc = (int)nc64;
  // contigs: cstart cend sbeg ; cscaf (int32); clen and boff go to the GDB's own arrays
  ENSURE(ctx->fa_ctg, sizeof(int64_t) * 3 * (nc + 1) + sizeof(int32_t) * (nc + 1));
  int64_t *cstart = P<int64_t>(ctx->fa_ctg), *cend = cstart + (nc + 1), *sbeg = cend + (nc + 1);
  int32_t *cscaf = (int32_t *)(sbeg + (nc + 1));
  ENSURE(ctx->dclen, sizeof(int64_t) * (nc + 1));
  ENSURE(ctx->dboff, sizeof(int64_t) * (nc + 1));
  ENSURE(ctx->fa_tmp, sizeof(int64_t) * std::max(scan_tmp_elems(R), scan_tmp_elems(nc)));
  int64_t *dclen = P<int64_t>(ctx->dclen), *dboff = P<int64_t>(ctx->dboff);
  CK(fa_scaffolds(sstart, nh, rs, R, sr, nsplit, trail, hoff, scf4, cstart, cend, cscaf, st));
  if (R > 0) {
    CK(fa_splits(rs, re, R, isp, sr, rscaf, cstart, cend, cscaf, st));
    LAUNCHED(1);
  }
  CK(fa_contigs(nc, cstart, cend, cscaf, sstart, dclen, sbeg, dboff, status, st));
  CK(exclusive_scan<int64_t>(dboff, dboff, nc, P<int64_t>(ctx->fa_tmp), dboff + nc, st));
  LAUNCHED(5);
  TRY(fetch(ctx, h + 6, dboff + nc, 1));
  CK(cudaStreamSynchronize(st));
  const int64_t nbps = h[6];
  ENSURE(ctx->bps, (size_t)((nbps + 3) / 4 * 4) + 16);
  CK(fa_pack(seq, nc, dboff, cstart, dclen, P<uint8_t>(ctx->bps), st));
  CK(cudaEventRecord(ctx->fa_ev[2], st));
  LAUNCHED(1);

  // host tables
  std::vector<int64_t> clen(nc), boff(nc);
  ctx->h_sbeg.resize(nc);
  ctx->h_scaf.resize(nc);
  ctx->h_scf4.resize(4 * (size_t)nh);
  ctx->h_headers.resize(hdrtot);
  TRY(fetch(ctx, clen.data(), dclen, nc));
  TRY(fetch(ctx, boff.data(), dboff, nc));
  TRY(fetch(ctx, ctx->h_sbeg.data(), sbeg, nc));
  TRY(fetch(ctx, ctx->h_scaf.data(), cscaf, nc));
  TRY(fetch(ctx, ctx->h_scf4.data(), scf4, 4 * (int64_t)nh));
  TRY(fetch(ctx, ctx->h_headers.data(), ctx->fa_hbytes.p, hdrtot));
  TRY(fetch(ctx, hs, status, FA_NSTATUS + 256));
  CK(cudaStreamSynchronize(st));
  for (int v = 0; v < 4; v++) {
    unsigned long long c = 0;
    for (int b = 0; b < 64; b++) c += hs[FA_NSTATUS + 4 * b + v];
    ctx->base_count[v] = (int64_t)c;
  }
  ctx->base_count[0] += (int64_t)hs[FA_FILL];
  TRY(gdb_tables(ctx, nc, clen.data(), boff.data(), nbps));
  const int64_t seqtot = ctx->base_count[0] + ctx->base_count[1] + ctx->base_count[2] + ctx->base_count[3];
  // GDB.freq as Create_GDB sets it (lib/GDB.c:1083-1086)
  for (int v = 0; v < 4; v++) ctx->base_freq[v] = (float)((1. * ctx->base_count[v]) / seqtot);
  ctx->freq_set = true;
  if (sizes6) {
    sizes6[0] = nh;
    sizes6[1] = nc;
    sizes6[2] = nbps;
    sizes6[3] = hdrtot;
    sizes6[4] = (int64_t)hs[FA_MAXCTG];
    sizes6[5] = seqtot;
  }
  return PGA_OK;
}

}  // namespace

int pga_gdb_ingest_fasta(pga_ctx *ctx, const char *text, int64_t nbytes, int nthr, int64_t *sizes6) {
  if (!ctx || nbytes < 0 || (nbytes > 0 && !text)) return PGA_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  gdb_reset(ctx);
  if (nbytes == 0) return fail(ctx, PGA_ERR_ARG, "input is empty");
  if (text[0] != '>') return fail(ctx, PGA_ERR_ARG, "first header is missing");
  if (text[nbytes - 1] != '\n') return fail(ctx, PGA_ERR_ARG, "last line does not end with new-line");
  for (cudaEvent_t &e : ctx->fa_ev)
    if (!e) CK(cudaEventCreate(&e));
  ENSURE(ctx->fa_text, (size_t)nbytes + 64);
  CK(cudaEventRecord(ctx->fa_ev[0], ctx->st));
  CK(cudaMemcpyAsync(ctx->fa_text.p, text, nbytes, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemsetAsync(P<uint8_t>(ctx->fa_text) + nbytes, 0, 64, ctx->st));
  CK(cudaEventRecord(ctx->fa_ev[1], ctx->st));
  int r = ingest_device(ctx, nbytes, nthr, sizes6);
  if (r != PGA_OK) return r;
  CK(cudaEventElapsedTime(&ctx->ingest_ms[0], ctx->fa_ev[0], ctx->fa_ev[1]));
  CK(cudaEventElapsedTime(&ctx->ingest_ms[1], ctx->fa_ev[1], ctx->fa_ev[2]));
  ctx->have_gdb = true;
  ctx->have_scaffolds = true;
  ctx->ingest_nthr = nthr;
  return PGA_OK;
}

int pga_gdb_ingest_times(const pga_ctx *ctx, float *ms2) {
  if (!ctx || !ms2 || !ctx->have_scaffolds) return PGA_ERR_ARG;
  ms2[0] = ctx->ingest_ms[0];
  ms2[1] = ctx->ingest_ms[1];
  return PGA_OK;
}

int pga_gdb_copy(pga_ctx *ctx, uint8_t *bps, int64_t *contigs4, int64_t *scaffolds4, char *headers,
                 int64_t *counts4) {
  if (!ctx || !ctx->have_scaffolds) return PGA_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  if (bps && ctx->bps_bytes > 0) {
    CK(cudaMemcpyAsync(bps, ctx->bps.p, ctx->bps_bytes, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
  if (contigs4)
    for (int c = 0; c < ctx->ncontig; c++) {
      contigs4[4 * c + 0] = ctx->clen[c];
      contigs4[4 * c + 1] = ctx->boff[c];
      contigs4[4 * c + 2] = ctx->h_sbeg[c];
      contigs4[4 * c + 3] = ctx->h_scaf[c];
    }
  if (scaffolds4) std::copy(ctx->h_scf4.begin(), ctx->h_scf4.end(), scaffolds4);
  if (headers) std::copy(ctx->h_headers.begin(), ctx->h_headers.end(), headers);
  if (counts4)
    for (int v = 0; v < 4; v++) counts4[v] = ctx->base_count[v];
  return PGA_OK;
}

int pga_gdb_write(pga_ctx *ctx, const char *tpath, const char *program, const char *version, const char *command,
                  const char *srcpath) {
  if (!ctx || !ctx->have_scaffolds || !tpath || !program || !version || !command || !srcpath) return PGA_ERR_ARG;
  std::vector<uint8_t> bps(ctx->bps_bytes);
  std::vector<int64_t> ctg(4 * (size_t)ctx->ncontig);
  int r = pga_gdb_copy(ctx, bps.data(), ctg.data(), nullptr, nullptr, nullptr);
  if (r != PGA_OK) return r;
  r = pga_write_1gdb(tpath, program, version, command, srcpath, ctx->base_freq, (int)(ctx->h_scf4.size() / 4),
                     ctx->h_scf4.data(), ctx->h_headers.data(), (int64_t)ctx->h_headers.size(), ctx->ncontig,
                     ctg.data(), bps.data(), ctx->bps_bytes);
  if (r != PGA_OK) return fail(ctx, r, "cannot write %s or its .bps", tpath);
  return PGA_OK;
}

int pga_record_sizing(const pga_ctx *ctx, int *posb, int *ctgb, int *rsize) {
  if (!ctx || !ctx->have_gdb) return PGA_ERR_ARG;
  if (posb) *posb = ctx->posb;
  if (ctgb) *ctgb = ctx->ctgb;
  if (rsize) *rsize = ctx->rsize;
  return PGA_OK;
}

int pga_extract_to_records(pga_ctx *ctx, int num_workers, int worker_id, uint8_t **records, int64_t *count) {
  if (!ctx || !ctx->have_gdb || !records || !count || num_workers < 1 || worker_id < 0 ||
      worker_id >= num_workers)
    return PGA_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  *records = nullptr;
  *count = 0;
  // Contig split by cumulative bases (compute_work_split, src/work_split.c:3-26).
  int64_t total = 0;
  for (int r = 0; r < ctx->ncontig; r++) total += ctx->clen[r];
  std::vector<int> split(num_workers + 1, 0);
  {
    int64_t so_far = 0, next = total / num_workers;
    int nw = 1;
    for (int r = 0; r < ctx->ncontig; r++) {
      so_far += ctx->clen[r];
      while (so_far >= next && nw < num_workers) {
        split[nw] = r + 1;
        nw += 1;
        next = (total * nw) / num_workers;
      }
    }
    split[num_workers] = ctx->ncontig;
  }
  int rbeg = split[worker_id], rend = split[worker_id + 1];
  int tbeg = 0, tend = 0;
  while (tbeg < ctx->ntiles && ctx->h_tile_ctg[tbeg] < rbeg) tbeg++;
  tend = tbeg;
  while (tend < ctx->ntiles && ctx->h_tile_ctg[tend] < rend) tend++;
  int nt = tend - tbeg;
  int64_t nthr = (int64_t)nt * EXT_THREADS;
  ENSURE(ctx->u64tmp, 64);
  ENSURE(ctx->io2, sizeof(uint64_t) * (nthr + 1) + 64);
  ENSURE(ctx->scan_tmp, sizeof(uint64_t) * scan_tmp_elems(nthr + 1) + 64);
  uint32_t *cnt32 = P<uint32_t>(ctx->hist);
  ENSURE(ctx->hist, sizeof(uint32_t) * std::max<int64_t>(NPREFIX + 1, nthr + 1));
  cnt32 = P<uint32_t>(ctx->hist);
  uint64_t *off = P<uint64_t>(ctx->io2);
  uint64_t total_rec = 0;
  if (nt > 0) {
    const int32_t *tc = P<int32_t>(ctx->tile_ctg) + tbeg;
    const int64_t *tj = P<int64_t>(ctx->tile_j0) + tbeg;
    launch_extract(EXT_COUNT, nt, ctx->st, P<uint8_t>(ctx->bps), P<int64_t>(ctx->dclen), P<int64_t>(ctx->dboff),
                   tc, tj, ctx->ctgb, cnt32, nullptr, nullptr, nullptr, nullptr);
    LAUNCHED(1);
    CK(cudaGetLastError());
    // widen the counts to 64 bits for the offsets scan
    std::vector<uint32_t> hc(nthr);
    CK(cudaMemcpyAsync(hc.data(), cnt32, sizeof(uint32_t) * nthr, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    std::vector<uint64_t> ho(nthr);
    for (int64_t i = 0; i < nthr; i++) {
      ho[i] = total_rec;
      total_rec += hc[i];
    }
    int r = check_records_fit(ctx, (int64_t)total_rec);
    if (r) return r;
    CK(cudaMemcpyAsync(off, ho.data(), sizeof(uint64_t) * nthr, cudaMemcpyHostToDevice, ctx->st));
    ENSURE(ctx->rec2, sizeof(Rec) * total_rec + 16);
    launch_extract(EXT_WRITE, nt, ctx->st, P<uint8_t>(ctx->bps), P<int64_t>(ctx->dclen), P<int64_t>(ctx->dboff),
                   tc, tj, ctx->ctgb, nullptr, off, P<Rec>(ctx->rec2), nullptr, nullptr);
    LAUNCHED(1);
    CK(cudaGetLastError());
  }
  size_t bytes = (size_t)total_rec * ctx->rsize;
  uint8_t *h = (uint8_t *)malloc(bytes + 1);
  if (!h) return fail(ctx, PGA_ERR_NOMEM, "malloc(%zu)", bytes + 1);
  if (total_rec > 0) {
    int r = ensure(ctx, ctx->io, bytes + 16);
    if (r) {
      free(h);
      return r;
    }
    k_records_out<<<grid_for(total_rec, 256), 256, 0, ctx->st>>>(P<Rec>(ctx->rec2), nullptr, total_rec, ctx->posb,
                                                                  ctx->ctgb, P<uint8_t>(ctx->io));
    LAUNCHED(1);
    cudaError_t e = cudaMemcpyAsync(h, ctx->io.p, bytes, cudaMemcpyDeviceToHost, ctx->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
    if (e != cudaSuccess) {
      free(h);
      return fail(ctx, PGA_ERR_CUDA, "extract copy: %s", cudaGetErrorString(e));
    }
  }
  *records = h;
  *count = (int64_t)total_rec;
  return PGA_OK;
}

int pga_sort_records(pga_ctx *ctx, uint8_t *records, int64_t count, int posb, int ctgb) {
  if (!ctx || count < 0 || (count > 0 && !records) || posb < 1 || posb > 4 || ctgb < 1 || ctgb > 2)
    return PGA_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  int r = index_from_host(ctx, records, count, posb, ctgb);
  if (r) return r;
  int rs = 12 + posb + ctgb;
  ENSURE(ctx->lcp, (size_t)count + 16);
  if (count > 0) {
    k_lcp<<<grid_for(count, 256), 256, 0, ctx->st>>>(P<Rec>(ctx->rec), count, P<uint8_t>(ctx->lcp));
    k_records_out<<<grid_for(count, 256), 256, 0, ctx->st>>>(P<Rec>(ctx->rec), P<uint8_t>(ctx->lcp), count, posb,
                                                              ctgb, P<uint8_t>(ctx->io));
    LAUNCHED(2);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(records, ctx->io.p, (size_t)count * rs, cudaMemcpyDeviceToHost, ctx->st));
  }
  CK(cudaStreamSynchronize(ctx->st));
  ctx->have_index = false;
  return PGA_OK;
}

int pga_recalc_lcps(pga_ctx *ctx, uint8_t *records, int64_t count, int posb, int ctgb) {
  if (!ctx || count < 0 || (count > 0 && !records) || posb < 1 || posb > 4 || ctgb < 1 || ctgb > 2)
    return PGA_ERR_ARG;
  if (count == 0) return PGA_OK;
  CK(cudaSetDevice(ctx->device));
  int r = check_records_fit(ctx, count);
  if (r) return r;
  const int rs = 12 + posb + ctgb;
  ENSURE(ctx->io, (size_t)count * rs + 16);
  ENSURE(ctx->rec, sizeof(Rec) * (size_t)count + 16);
  ENSURE(ctx->lcp, (size_t)count + 16);
  CK(cudaMemcpyAsync(ctx->io.p, records, (size_t)count * rs, cudaMemcpyHostToDevice, ctx->st));
  k_records_in<<<grid_for(count, 256), 256, 0, ctx->st>>>(P<uint8_t>(ctx->io), count, posb, ctgb, P<Rec>(ctx->rec),
                                                           P<uint8_t>(ctx->lcp));
  k_lcp<<<grid_for(count, 256), 256, 0, ctx->st>>>(P<Rec>(ctx->rec), count, P<uint8_t>(ctx->lcp));
  k_records_out<<<grid_for(count, 256), 256, 0, ctx->st>>>(P<Rec>(ctx->rec), P<uint8_t>(ctx->lcp), count, posb, ctgb,
                                                            P<uint8_t>(ctx->io));
  LAUNCHED(3);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(records, ctx->io.p, (size_t)count * rs, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->have_index = false;
  return PGA_OK;
}

int pga_build_kmer_adapter(pga_ctx *ctx, const uint8_t *records, int64_t count, int posb, int ctgb,
                           uint8_t *entries, int64_t *cum, int64_t *largest) {
  if (!ctx || count < 0 || (count > 0 && (!records || !entries)) || !cum || posb < 1 || posb > 4 || ctgb < 1 ||
      ctgb > 2)
    return PGA_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  int r = check_records_fit(ctx, count);
  if (r) return r;
  int rs = 12 + posb + ctgb, eb = 9 + posb + ctgb;
  ENSURE(ctx->io, (size_t)count * rs + 16);
  ENSURE(ctx->rec, sizeof(Rec) * (size_t)count + 16);
  ENSURE(ctx->lcp, (size_t)count + 16);
  ENSURE(ctx->ent, (size_t)count * eb + 16);
  ENSURE(ctx->cum, sizeof(int64_t) * NPREFIX);
  ENSURE(ctx->hist, sizeof(uint32_t) * (NPREFIX + 1));
  ENSURE(ctx->start, sizeof(uint32_t) * (NPREFIX + 1));
  ENSURE(ctx->maxrun, 16);
  // The records are already sorted: their prefixes' histogram scan gives the table.
  CK(cudaMemsetAsync(ctx->hist.p, 0, sizeof(uint32_t) * NPREFIX, ctx->st));
  if (count > 0) {
    CK(cudaMemcpyAsync(ctx->io.p, records, (size_t)count * rs, cudaMemcpyHostToDevice, ctx->st));
    k_records_in<<<grid_for(count, 256), 256, 0, ctx->st>>>(P<uint8_t>(ctx->io), count, posb, ctgb, P<Rec>(ctx->rec), P<uint8_t>(ctx->lcp));
    k_prefix_hist<<<grid_for(count, 256), 256, 0, ctx->st>>>(P<Rec>(ctx->rec), count, P<uint32_t>(ctx->hist));
    LAUNCHED(2);
  }
  ctx->posb = posb;
  ctx->ctgb = ctgb;
  ctx->rsize = rs;
  ctx->nrec = count;
  int64_t tot = 0;
  r = scan_hist(ctx, &tot);
  if (r) return r;
  // LCP bytes are the records' own (byte 0), not recomputed.
  if (count > 0) {
    k_entries<<<grid_for(count, 256), 256, 0, ctx->st>>>(P<Rec>(ctx->rec), P<uint8_t>(ctx->lcp), count, posb, ctgb,
                                                         P<uint8_t>(ctx->ent));
    LAUNCHED(1);
  }
  CK(cudaMemsetAsync(ctx->maxrun.p, 0, 4, ctx->st));
  k_prefix_table<<<NPREFIX / 256, 256, 0, ctx->st>>>(P<uint32_t>(ctx->start), P<int64_t>(ctx->cum),
                                                     P<uint32_t>(ctx->maxrun));
  LAUNCHED(1);
  CK(cudaGetLastError());
  if (count > 0) CK(cudaMemcpyAsync(entries, ctx->ent.p, (size_t)count * eb, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaMemcpyAsync(cum, ctx->cum.p, sizeof(int64_t) * NPREFIX, cudaMemcpyDeviceToHost, ctx->st));
  uint32_t mr = 0;
  CK(cudaMemcpyAsync(&mr, ctx->maxrun.p, 4, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (largest) *largest = mr;
  ctx->have_index = true;
  ctx->have_entries = true;
  ctx->largest = mr;
  return PGA_OK;
}

int pga_self_adaptamer_merge(pga_ctx *ctx, const uint8_t *entries, const int64_t *cum, int64_t count, int posb,
                             int ctgb, int freq, int ncontig, uint8_t **nseeds, int64_t *nlen, uint8_t **cseeds,
                             int64_t *clen_out, int64_t *nbuck, int64_t *cbuck) {
  if (!ctx || count < 0 || (count > 0 && !entries) || !cum || !nseeds || !nlen || !cseeds || !clen_out ||
      posb < 1 || posb > 4 || ctgb < 1 || ctgb > 2 || freq < 1 || ncontig < 1)
    return PGA_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  int r = check_records_fit(ctx, count);
  if (r) return r;
  *nseeds = *cseeds = nullptr;
  *nlen = *clen_out = 0;
  int eb = 9 + posb + ctgb;
  ENSURE(ctx->io, (size_t)count * eb + 16);
  ENSURE(ctx->cum, sizeof(int64_t) * NPREFIX);
  ENSURE(ctx->rec, sizeof(Rec) * (size_t)count + 16);
  ENSURE(ctx->lcp, (size_t)count + 16);
  if (count > 0) CK(cudaMemcpyAsync(ctx->io.p, entries, (size_t)count * eb, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemcpyAsync(ctx->cum.p, cum, sizeof(int64_t) * NPREFIX, cudaMemcpyHostToDevice, ctx->st));
  k_entries_in<<<NPREFIX / 256, 256, 0, ctx->st>>>(P<uint8_t>(ctx->io), P<int64_t>(ctx->cum), count, posb, ctgb,
                                                   P<Rec>(ctx->rec), P<uint8_t>(ctx->lcp));
  LAUNCHED(1);
  CK(cudaGetLastError());
  ctx->posb = posb;
  ctx->ctgb = ctgb;
  ctx->nrec = count;
  int saved_nc = ctx->ncontig;
  ctx->ncontig = ncontig;
  r = run_merge(ctx, freq);
  if (r) {
    ctx->ncontig = saved_nc;
    return r;
  }
  int sb = 1 + 2 * (posb + ctgb);
  uint8_t *hs[2] = {nullptr, nullptr};
  int64_t *bk[2] = {nbuck, cbuck};
  for (int u = 0; u < 2; u++) {
    hs[u] = (uint8_t *)malloc((size_t)ctx->nseed[u] * sb + 1);
    if (!hs[u]) {
      free(hs[0]);
      ctx->ncontig = saved_nc;
      return fail(ctx, PGA_ERR_NOMEM, "malloc seeds");
    }
    r = copy_seeds(ctx, u, hs[u], bk[u]);
    if (r) {
      free(hs[0]);
      free(hs[1]);
      ctx->ncontig = saved_nc;
      return r;
    }
  }
  ctx->ncontig = saved_nc;
  *nseeds = hs[0];
  *cseeds = hs[1];
  *nlen = ctx->nseed[0] * sb;
  *clen_out = ctx->nseed[1] * sb;
  return PGA_OK;
}

int pga_reimport_sort(pga_ctx *ctx, const uint8_t *seeds, int64_t len, int posb, int ctgb, int comp, int ncontig,
                      int64_t amxpos, int dbyte, uint8_t *out, int64_t *panel_off) {
  if (!ctx || len < 0 || (len > 0 && (!seeds || !out)) || !panel_off || posb < 1 || posb > 4 || ctgb < 1 ||
      ctgb > 2 || (comp != 0 && comp != 1) || ncontig < 1 || dbyte < 1 || dbyte > 4 || amxpos < 0)
    return PGA_ERR_ARG;
  int sb = 1 + 2 * (posb + ctgb);
  if (len % sb != 0) return fail(ctx, PGA_ERR_ARG, "seed bytes not a whole number of seeds");
  CK(cudaSetDevice(ctx->device));
  int64_t n = len / sb;
  if (n >= (int64_t)0xffffffffLL) return fail(ctx, PGA_ERR_LIMIT, "too many seeds");
  ENSURE(ctx->io, (size_t)len + 16);
  ENSURE(ctx->seed[comp], sizeof(Seed) * (size_t)n + 16);
  if (n > 0) {
    CK(cudaMemcpyAsync(ctx->io.p, seeds, (size_t)n * sb, cudaMemcpyHostToDevice, ctx->st));
    k_seeds_in<<<grid_for(n, 256), 256, 0, ctx->st>>>(P<uint8_t>(ctx->io), n, posb, ctgb, P<Seed>(ctx->seed[comp]));
    LAUNCHED(1);
  }
  ctx->nseed[comp] = n;
  ctx->seeds_consumed[comp] = false;
  int r = run_diag(ctx, comp, ncontig, amxpos, dbyte, ctgb);
  if (r) return r;
  return copy_diag(ctx, comp, ncontig, out, panel_off);
}

namespace {

// The two-level sort of the records of extraction tiles [tile0, tile0 +
// ntiles) into ctx->rec, with the prefix table (start) of those records;
// seqtot (the tiles' bases) sizes the digit.
int sort_tiles(pga_ctx *ctx, int tile0, int ntiles, int64_t seqtot) {
  const int dbits = ctx->digit_bits ? ctx->digit_bits : digit_bits_for(seqtot - seqtot / 5), dshift = 24 - dbits;
  const int64_t ndigit = (int64_t)1 << dbits;
  ENSURE(ctx->hist, sizeof(uint32_t) * (ndigit + 1));
  ENSURE(ctx->start, sizeof(uint32_t) * (NPREFIX + 1));
  // digit starts (ndigit + 1), digit cursors (ndigit + 1), digits above DS_CAP
  // (ndigit) and above DS_CAP_MID (ndigit)
  ENSURE(ctx->coarse, sizeof(uint32_t) * (4 * (size_t)ndigit + 2));
  uint32_t *dstart = P<uint32_t>(ctx->coarse), *dcur = dstart + (ndigit + 1), *qdig = dcur + (ndigit + 1),
           *qdig2 = qdig + ndigit;
  uint32_t *hist = P<uint32_t>(ctx->hist), *start = P<uint32_t>(ctx->start);
  const uint8_t *bps = P<uint8_t>(ctx->bps);
  const int64_t *cl = P<int64_t>(ctx->dclen), *bo = P<int64_t>(ctx->dboff);
  const int32_t *tc = P<int32_t>(ctx->tile_ctg) + tile0;
  const int64_t *tj = P<int64_t>(ctx->tile_j0) + tile0;
  stage_begin(ctx, ST_EXTRACT_HIST);
  CK(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * (ndigit + 1), ctx->st));
  if (ntiles > 0) {
    launch_extract(EXT_HIST, ntiles, ctx->st, bps, cl, bo, tc, tj, ctx->ctgb, nullptr, nullptr, nullptr, hist,
                   nullptr, dshift);
    LAUNCHED(1);
  }
  stage_end(ctx, ST_EXTRACT_HIST);
  CK(cudaGetLastError());
  stage_begin(ctx, ST_SCAN);
  ENSURE(ctx->scan_tmp, sizeof(uint32_t) * scan_tmp_elems(ndigit + 1));
  CK(exclusive_scan<uint32_t>(hist, dstart, ndigit + 1, P<uint32_t>(ctx->scan_tmp), (uint32_t *)nullptr, ctx->st));
  LAUNCHED(3);
  CK(cudaMemcpyAsync(dcur, dstart, sizeof(uint32_t) * ndigit, cudaMemcpyDeviceToDevice, ctx->st));
  CK(cudaMemcpyAsync(start + NPREFIX, dstart + ndigit, sizeof(uint32_t), cudaMemcpyDeviceToDevice, ctx->st));
  uint32_t total = 0;
  CK(cudaMemcpyAsync(&total, dstart + ndigit, 4, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  stage_end(ctx, ST_SCAN);
  const int64_t n = total;
  int r = check_records_fit(ctx, n);
  if (r) return r;
  ctx->nrec = n;
  ENSURE(ctx->rec, sizeof(Rec) * (size_t)n + 16);
  // level 1: every record into its digit's region
  stage_begin(ctx, ST_EXTRACT_SCATTER);
  if (ntiles > 0) {
    launch_extract(EXT_DIGIT, ntiles, ctx->st, bps, cl, bo, tc, tj, ctx->ctgb, nullptr, nullptr,
                   P<Rec>(ctx->rec), nullptr, dcur, dshift);
    LAUNCHED(1);
  }
  stage_end(ctx, ST_EXTRACT_SCATTER);
  CK(cudaGetLastError());
  // level 2: each digit sorted in shared memory; larger digits grouped by
  // prefix in global memory and their buckets queued
  stage_begin(ctx, ST_BUCKET);
  ENSURE(ctx->qmed, sizeof(uint32_t) * NPREFIX);
  ENSURE(ctx->qbig, sizeof(uint32_t) * NPREFIX);
  ENSURE(ctx->qcount, sizeof(uint32_t) * 8);
  CK(cudaMemsetAsync(ctx->qcount.p, 0, sizeof(uint32_t) * 8, ctx->st));
  uint32_t *qc = P<uint32_t>(ctx->qcount);
  CK(launch_digit_sort(DS_CAP, (int)ndigit, DS_THREADS, ctx->st, P<Rec>(ctx->rec), dstart, start, nullptr, qdig,
                       qc + 4, dshift));
  LAUNCHED(1);
  CK(cudaGetLastError());
  uint32_t q[8];
  CK(cudaMemcpyAsync(q, qc, sizeof(q), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (q[4] > 0) {
    CK(launch_digit_sort(DS_CAP_MID, (int)q[4], DS_MID_THREADS, ctx->st, P<Rec>(ctx->rec), dstart, start, qdig,
                         qdig2, qc + 5, dshift));
    LAUNCHED(1);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(q, qc, sizeof(q), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
  if (q[5] > 0) {
    // scratch for the big digits only: digit i of the list at toff[i]
    std::vector<uint32_t> big(q[5]), hd(ndigit + 1);
    CK(cudaMemcpyAsync(big.data(), qdig2, sizeof(uint32_t) * q[5], cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(hd.data(), dstart, sizeof(uint32_t) * (ndigit + 1), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    std::vector<int64_t> toff(q[5] + 1, 0);
    for (uint32_t i = 0; i < q[5]; i++) toff[i + 1] = toff[i] + (hd[big[i] + 1] - hd[big[i]]);
    ENSURE(ctx->rec2, sizeof(Rec) * (size_t)toff[q[5]] + 16);
    ENSURE(ctx->u64tmp, sizeof(int64_t) * (q[5] + 1));
    CK(cudaMemcpyAsync(ctx->u64tmp.p, toff.data(), sizeof(int64_t) * (q[5] + 1), cudaMemcpyHostToDevice, ctx->st));
    k_big_digit<<<q[5], BD_THREADS, 0, ctx->st>>>(P<Rec>(ctx->rec), dstart, start, qdig2, P<int64_t>(ctx->u64tmp),
                                                  P<Rec>(ctx->rec2), P<uint32_t>(ctx->qmed), P<uint32_t>(ctx->qbig),
                                                  qc, dshift);
    LAUNCHED(1);
    CK(cudaGetLastError());
  }
  r = sort_queued(ctx);
  if (r) return r;
  stage_end(ctx, ST_BUCKET);
  return PGA_OK;
}

}  // namespace

int pga_index_build(pga_ctx *ctx, int want_entries, int64_t *count) {
  if (!ctx || !ctx->have_gdb) return PGA_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  // digit width (records ~ 0.8 per base)
  int64_t seqtot = 0;
  for (int c = 0; c < ctx->ncontig; c++) seqtot += ctx->clen[c];
  int r = sort_tiles(ctx, 0, ctx->ntiles, seqtot);
  if (r) return r;
  r = finish_index(ctx, want_entries != 0);
  if (r) return r;
  if (count) *count = ctx->nrec;
  return PGA_OK;
}

namespace {

// pga_target_create; with keep, the context keeps its GDB and index.
int target_create(pga_ctx *ctx, pga_target **out, bool keep) {
  if (!ctx || !out) return PGA_ERR_ARG;
  *out = nullptr;
  if (!ctx->have_scaffolds || !ctx->have_index)
    return fail(ctx, PGA_ERR_ARG, "a target needs an ingested GDB (pga_gdb_ingest_fasta) and its index (pga_index_build)");
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->st));
  pga_target *t = new (std::nothrow) pga_target();
  if (!t) return fail(ctx, PGA_ERR_NOMEM, "host allocation");
  t->device = ctx->device;
  t->ncontig = ctx->ncontig;
  t->ctgb = ctx->ctgb;
  t->nthr = ctx->ingest_nthr;
  t->bps_bytes = ctx->bps_bytes;
  t->nrec = ctx->nrec;
  t->clen = ctx->clen;
  t->boff = ctx->boff;
  t->sbeg = ctx->h_sbeg;
  t->scf4 = ctx->h_scf4;
  t->scaf = ctx->h_scaf;
  t->headers = ctx->h_headers;
  for (int v = 0; v < 4; v++) t->base_count[v] = ctx->base_count[v];
  // the target owns its buffers (it may outlive the context): each is copied
  // out of the context's arena, whose copy is then freed
  struct {
    DBuf *from, *to;
  } mv[3] = {{&ctx->bps, &t->bps}, {&ctx->rec, &t->rec}, {&ctx->start, &t->start}};
  for (auto &m : mv) {
    const size_t n = m.from->cap;
    cudaError_t e = cudaMalloc(&m.to->p, n);
    if (e != cudaSuccess) {
      cudaGetLastError();
      m.to->p = nullptr;
      ctx->arena.trim();
      e = cudaMalloc(&m.to->p, n);
      if (e != cudaSuccess) m.to->p = nullptr;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(m.to->p, m.from->p, n, cudaMemcpyDeviceToDevice, ctx->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      if (m.to->p) cudaFree(m.to->p);
      m.to->p = nullptr;
      pga_target_destroy(t);
      return fail(ctx, PGA_ERR_NOMEM, "target buffer of %zu bytes: %s", n, cudaGetErrorString(e));
    }
    m.to->cap = n;
    if (!keep) {
      ctx->arena.release(m.from->p);
      m.from->p = nullptr;
      m.from->cap = 0;
    }
  }
  if (!keep) gdb_reset(ctx);
  *out = t;
  return PGA_OK;
}

int target_upload(pga_ctx *ctx, DBuf &b, const void *src, size_t bytes) {
  b.cap = bytes + 16;
  cudaError_t e = cudaMalloc(&b.p, b.cap);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    b.cap = 0;
    return fail(ctx, PGA_ERR_NOMEM, "target cache buffer of %zu bytes: %s", bytes, cudaGetErrorString(e));
  }
  if (bytes > 0 && src) CK(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return PGA_OK;
}

// The target's table of Local_Alignment calls from the context's log of its
// own run: every logged call whose trace was kept, once per distinct input,
// in an open-addressing table of twice as many slots (a power of two).
int build_memo(pga_ctx *ctx, pga_target *t) {
  unsigned long long ctr[2];
  CK(cudaMemcpyAsync(ctr, ctx->mlog_ctr.p, 16, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  const int64_t e = std::min<int64_t>((int64_t)ctr[0], ctx->cap_calls);
  const int64_t tb = std::min<int64_t>((int64_t)ctr[1], ctx->cap_bytes);
  std::vector<uint32_t> lk(MEMO_KEY * (size_t)e);
  std::vector<int32_t> lv(MEMO_VAL * (size_t)e);
  std::vector<int64_t> lt(e);
  if (e > 0) {
    CK(cudaMemcpyAsync(lk.data(), ctx->mlog_key.p, 4 * lk.size(), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(lv.data(), ctx->mlog_val.p, 4 * lv.size(), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(lt.data(), ctx->mlog_toff.p, 8 * lt.size(), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
  const MemoTable T = memo_table(lk.data(), lv.data(), lt.data(), e);
  pga_target::Memo &M = t->memo;
  int r;
  if ((r = target_upload(ctx, M.key, T.key.data(), 4 * T.key.size()))) return r;
  if ((r = target_upload(ctx, M.val, T.val.data(), 4 * T.val.size()))) return r;
  if ((r = target_upload(ctx, M.toff, T.toff.data(), 8 * T.toff.size()))) return r;
  if ((r = target_upload(ctx, M.trace, nullptr, (size_t)tb))) return r;
  if (tb > 0) CK(cudaMemcpyAsync(M.trace.p, ctx->mlog_trace.p, (size_t)tb, cudaMemcpyDeviceToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  M.cap = T.cap;
  M.entries = T.entries;
  M.spec = ctx->spec_host;
  M.ave_path = ctx->ave_path_host;
  M.valid = true;
  return PGA_OK;
}

}  // namespace

int pga_target_create(pga_ctx *ctx, pga_target **out) { return target_create(ctx, out, false); }

int pga_target_create_reuse(pga_ctx *ctx, int freq, pga_target **out) {
  if (!ctx || !out || freq < 1) return PGA_ERR_ARG;
  pga_target *t = nullptr;
  int r = target_create(ctx, &t, true);
  if (r) return r;
  // the target's own run: once to count its calls, then again with every
  // call logged (and once more if the log was too small for the traces)
  r = run_merge(ctx, freq);
  int64_t nal = 0;
  if (!r) r = pga_align(ctx, &nal);
  ctx->cap_calls = ctx->align_work[2] + 1024;
  ctx->cap_bytes = 64 * ctx->cap_calls + (16 << 20);
  for (int attempt = 0; !r && attempt < 2; attempt++) {
    ctx->capture = true;
    r = pga_align(ctx, &nal);
    ctx->capture = false;
    if (r) break;
    unsigned long long ctr[2];
    CK(cudaMemcpyAsync(ctr, ctx->mlog_ctr.p, 16, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if ((int64_t)ctr[0] <= ctx->cap_calls && (int64_t)ctr[1] <= ctx->cap_bytes) break;
    ctx->cap_calls = (int64_t)ctr[0] + 1024;
    ctx->cap_bytes = (int64_t)ctr[1] + (16 << 20);
  }
  if (!r) r = build_memo(ctx, t);
  ctx->capture = false;
  gdb_reset(ctx);
  if (r) {
    pga_target_destroy(t);
    return r;
  }
  *out = t;
  return PGA_OK;
}

void pga_target_destroy(pga_target *t) {
  if (!t) return;
  cudaSetDevice(t->device);
  for (DBuf *b : {&t->bps, &t->rec, &t->start})
    if (b->p) cudaFree(b->p);
  for (DBuf *b : {&t->memo.key, &t->memo.val, &t->memo.toff, &t->memo.trace})
    if (b->p) cudaFree(b->p);
  delete t;
}

int pga_target_info(const pga_target *t, int64_t *info4) {
  if (!t || !info4) return PGA_ERR_ARG;
  int64_t bases = 0;
  for (int64_t c : t->clen) bases += c;
  info4[0] = t->ncontig;
  info4[1] = bases;
  info4[2] = t->nrec;
  const size_t cache = t->memo.key.cap + t->memo.val.cap + t->memo.toff.cap + t->memo.trace.cap;
  info4[3] = (int64_t)(t->bps.cap + t->rec.cap + t->start.cap + cache);
  return PGA_OK;
}

int pga_align_reuse_stats(const pga_ctx *ctx, int64_t *stats4) {
  if (!ctx || !stats4) return PGA_ERR_ARG;
  for (int i = 0; i < 4; i++) stats4[i] = ctx->reuse_stats[i];
  return PGA_OK;
}

int pga_serve_load(pga_ctx *ctx, const pga_target *t, const char *query, int64_t nbytes, int want_entries,
                   int64_t *sizes6, int64_t *count) {
  if (!ctx || !t) return PGA_ERR_ARG;
  if (t->device != ctx->device) return fail(ctx, PGA_ERR_ARG, "target on device %d, context on %d", t->device, ctx->device);
  // the query's GDB, read with the target's gap threshold
  int r = pga_gdb_ingest_fasta(ctx, query, nbytes, t->nthr, nullptr);
  if (r) return r;
  ctx->have_gdb = ctx->have_scaffolds = false;
  const int qnc = ctx->ncontig, qnh = (int)(ctx->h_scf4.size() / 4);
  const int64_t nc64 = (int64_t)t->ncontig + qnc, nh64 = (int64_t)(t->scf4.size() / 4) + qnh;
  if (nc64 >= 32768) return fail(ctx, PGA_ERR_LIMIT, "%lld contigs: at most 32767 supported", (long long)nc64);
  if (nh64 >= 32768) return fail(ctx, PGA_ERR_LIMIT, "%lld scaffolds: at most 32767 supported", (long long)nh64);
  const int nc = (int)nc64;
  // GDB(target, query): the target's image followed by the query's, as the
  // ingest of the two texts one after the other lays it out
  const int64_t tb = t->bps_bytes, qb = ctx->bps_bytes, nb = tb + qb;
  ENSURE(ctx->io2, (size_t)((nb + 3) / 4 * 4) + 16);
  if (tb > 0) CK(cudaMemcpyAsync(ctx->io2.p, t->bps.p, tb, cudaMemcpyDeviceToDevice, ctx->st));
  if (qb > 0) CK(cudaMemcpyAsync(P<uint8_t>(ctx->io2) + tb, ctx->bps.p, qb, cudaMemcpyDeviceToDevice, ctx->st));
  CK(cudaMemsetAsync(P<uint8_t>(ctx->io2) + nb, 0, (size_t)((nb + 3) / 4 * 4) + 16 - nb, ctx->st));
  std::swap(ctx->bps, ctx->io2);
  std::vector<int64_t> clen(t->clen), boff(t->boff);
  for (int c = 0; c < qnc; c++) {
    clen.push_back(ctx->clen[c]);
    boff.push_back(ctx->boff[c] + tb);
  }
  const int64_t th = (int64_t)t->headers.size();
  std::vector<int64_t> sbeg(t->sbeg), scf4(t->scf4);
  std::vector<int32_t> scaf(t->scaf);
  sbeg.insert(sbeg.end(), ctx->h_sbeg.begin(), ctx->h_sbeg.end());
  for (int32_t s : ctx->h_scaf) scaf.push_back(s + (int32_t)(t->scf4.size() / 4));
  for (int j = 0; j < qnh; j++) {
    scf4.push_back(ctx->h_scf4[4 * j + 0] + t->ncontig);
    scf4.push_back(ctx->h_scf4[4 * j + 1] + t->ncontig);
    scf4.push_back(ctx->h_scf4[4 * j + 2]);
    scf4.push_back(ctx->h_scf4[4 * j + 3] + th);
  }
  std::vector<char> headers(t->headers);
  headers.insert(headers.end(), ctx->h_headers.begin(), ctx->h_headers.end());
  ctx->h_sbeg.swap(sbeg);
  ctx->h_scaf.swap(scaf);
  ctx->h_scf4.swap(scf4);
  ctx->h_headers.swap(headers);
  int64_t seqtot = 0, qbases = 0;
  for (int v = 0; v < 4; v++) {
    ctx->base_count[v] += t->base_count[v];
    seqtot += ctx->base_count[v];
  }
  // GDB.freq as Create_GDB sets it (lib/GDB.c:1083-1086)
  for (int v = 0; v < 4; v++) ctx->base_freq[v] = (float)((1. * ctx->base_count[v]) / seqtot);
  ctx->freq_set = true;
  for (int c = 0; c < qnc; c++) qbases += ctx->clen[c];
  ENSURE(ctx->dclen, sizeof(int64_t) * (nc + 1));
  ENSURE(ctx->dboff, sizeof(int64_t) * (nc + 1));
  CK(cudaMemcpyAsync(ctx->dclen.p, clen.data(), sizeof(int64_t) * nc, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemcpyAsync(ctx->dboff.p, boff.data(), sizeof(int64_t) * nc, cudaMemcpyHostToDevice, ctx->st));
  r = gdb_tables(ctx, nc, clen.data(), boff.data(), nb);
  if (r) return r;
  ctx->have_gdb = ctx->have_scaffolds = true;
  ctx->ingest_nthr = t->nthr;
  // the index: the query's records sorted alone (its tiles follow the
  // target's), then their union with the target's
  int q0 = 0;
  while (q0 < ctx->ntiles && ctx->h_tile_ctg[q0] < t->ncontig) q0++;
  r = sort_tiles(ctx, q0, ctx->ntiles - q0, qbases);
  if (r) return r;
  const int64_t nq = ctx->nrec, n = t->nrec + nq;
  r = check_records_fit(ctx, n);
  if (r) return r;
  if (t->ctgb > ctx->ctgb) return fail(ctx, PGA_ERR_ARG, "target contig width %d above the request's %d", t->ctgb, ctx->ctgb);
  ENSURE(ctx->rec2, sizeof(Rec) * (size_t)n + 16);
  if (n > 0) {
    k_union_rank<<<grid_for(n, 256), 256, 0, ctx->st>>>(P<Rec>(t->rec), P<uint32_t>(t->start), t->nrec, t->ctgb,
                                                        P<Rec>(ctx->rec), P<uint32_t>(ctx->start), nq, ctx->ctgb,
                                                        P<Rec>(ctx->rec2));
    LAUNCHED(1);
  }
  k_add_prefix_tables<<<grid_for(NPREFIX + 1, 256), 256, 0, ctx->st>>>(P<uint32_t>(ctx->start), P<uint32_t>(t->start));
  LAUNCHED(1);
  CK(cudaGetLastError());
  std::swap(ctx->rec, ctx->rec2);
  ctx->nrec = n;
  r = finish_index(ctx, want_entries != 0);
  if (r) return r;
  if (sizes6) {
    sizes6[0] = (int64_t)(ctx->h_scf4.size() / 4);
    sizes6[1] = nc;
    sizes6[2] = nb;
    sizes6[3] = (int64_t)ctx->h_headers.size();
    sizes6[4] = ctx->maxctg;
    sizes6[5] = seqtot;
  }
  if (count) *count = n;
  ctx->reuse_t = t;  // its pair cache, if it has one, serves this GDB's alignment
  return PGA_OK;
}

int pga_index_write_gix(pga_ctx *ctx, const char *stem, int nparts) {
  if (!ctx || !stem || nparts < 1 || nparts > 1024) return PGA_ERR_ARG;
  if (!ctx->have_index || !ctx->have_entries)
    return fail(ctx, PGA_ERR_ARG, "no index with entries: call pga_index_build with want_entries = 1 first");
  CK(cudaSetDevice(ctx->device));
  // GIXmake's widths (notes/GIXmake_annotated.c:1966-1978): bytes for the
  // longest contig's positions, and for 2 x contigs
  auto width = [](int64_t range) {
    int b = 0;
    for (int64_t cum = 1; cum < range; cum *= 256) b++;
    return b;
  };
  const int postb = width(ctx->maxctg), contb = width(2 * (int64_t)ctx->ncontig);
  if (postb != ctx->posb || contb != ctx->ctgb)
    return fail(ctx, PGA_ERR_LIMIT, "GIXmake's entry widths (%d, %d) differ from the index's (%d, %d)", postb, contb,
                ctx->posb, ctx->ctgb);
  const int eb = 9 + ctx->posb + ctx->ctgb;
  std::vector<uint8_t> ent((size_t)ctx->nrec * eb + 1);
  std::vector<int64_t> cum((size_t)1 << 24);
  int64_t largest = 0;
  int r = pga_index_copy_entries(ctx, ent.data(), cum.data(), &largest);
  if (r != PGA_OK) return r;
  // contigs longest first, ties in contig order (GIXmake's LSORT under glibc's
  // merge sort, notes/GIXmake_annotated.c:1666-1671, 2037-2047)
  std::vector<int32_t> order(ctx->ncontig);
  for (int i = 0; i < ctx->ncontig; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return ctx->clen[x] > ctx->clen[y]; });
  r = pga_write_gix(stem, nparts, postb, contb, ctx->ncontig, order.data(), cum.data(), largest, ctx->nrec,
                    ent.data());
  if (r != PGA_OK) return fail(ctx, r, "cannot write %s.gix or its .ktab parts", stem);
  return PGA_OK;
}

int pga_index_copy_records(pga_ctx *ctx, uint8_t *records) {
  if (!ctx || !ctx->have_index || (!records && ctx->nrec > 0)) return PGA_ERR_ARG;
  int64_t n = ctx->nrec;
  ENSURE(ctx->io, (size_t)n * ctx->rsize + 16);
  if (n > 0) {
    k_records_out<<<grid_for(n, 256), 256, 0, ctx->st>>>(P<Rec>(ctx->rec), P<uint8_t>(ctx->lcp), n, ctx->posb,
                                                         ctx->ctgb, P<uint8_t>(ctx->io));
    LAUNCHED(1);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(records, ctx->io.p, (size_t)n * ctx->rsize, cudaMemcpyDeviceToHost, ctx->st));
  }
  CK(cudaStreamSynchronize(ctx->st));
  return PGA_OK;
}

int pga_index_copy_entries(pga_ctx *ctx, uint8_t *entries, int64_t *cum, int64_t *largest) {
  if (!ctx || !ctx->have_index || !ctx->have_entries) return PGA_ERR_ARG;
  int eb = 9 + ctx->posb + ctx->ctgb;
  if (entries && ctx->nrec > 0)
    CK(cudaMemcpyAsync(entries, ctx->ent.p, (size_t)ctx->nrec * eb, cudaMemcpyDeviceToHost, ctx->st));
  if (cum) CK(cudaMemcpyAsync(cum, ctx->cum.p, sizeof(int64_t) * NPREFIX, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (largest) *largest = ctx->largest;
  return PGA_OK;
}

int pga_merge(pga_ctx *ctx, int freq, int64_t *nseeds, int64_t *cseeds) {
  if (!ctx || !ctx->have_index || freq < 1) return PGA_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  int r = run_merge(ctx, freq);
  if (r) return r;
  if (nseeds) *nseeds = ctx->nseed[0];
  if (cseeds) *cseeds = ctx->nseed[1];
  return PGA_OK;
}

int pga_seeds_copy(pga_ctx *ctx, int comp, uint8_t *seeds, int64_t *buck) {
  if (!ctx || !ctx->have_seeds || (comp != 0 && comp != 1)) return PGA_ERR_ARG;
  if (ctx->seeds_released) return fail(ctx, PGA_ERR_ARG, "seeds were freed for the alignment; run pga_merge again");
  if (ctx->seeds_consumed[comp])
    return fail(ctx, PGA_ERR_ARG, "the unit's seeds were consumed by its diagonal sort; run pga_merge again");
  return copy_seeds(ctx, comp, seeds, buck);
}

int pga_seeds_load(pga_ctx *ctx, int comp, const uint8_t *seeds, int64_t len) {
  if (!ctx || !ctx->have_gdb || (comp != 0 && comp != 1) || len < 0 || (len > 0 && !seeds)) return PGA_ERR_ARG;
  const int sb = 1 + 2 * (ctx->posb + ctx->ctgb);
  if (len % sb != 0) return fail(ctx, PGA_ERR_ARG, "seed bytes not a whole number of seeds");
  const int64_t n = len / sb;
  if (n >= (int64_t)0xffffffffLL) return fail(ctx, PGA_ERR_LIMIT, "too many seeds");
  CK(cudaSetDevice(ctx->device));
  // both units are present from the first load on (the other one empty
  // until it is loaded too), as pga_merge leaves them
  if (!ctx->have_seeds || ctx->seeds_released || !ctx->seeds_loaded) {
    ctx->nseed[0] = ctx->nseed[1] = 0;
    ENSURE(ctx->seed[0], 16);
    ENSURE(ctx->seed[1], 16);
    ctx->seeds_loaded = true;
    ctx->have_diag[0] = ctx->have_diag[1] = false;
    ctx->seeds_consumed[0] = ctx->seeds_consumed[1] = false;
  }
  ENSURE(ctx->io, (size_t)len + 16);
  ENSURE(ctx->seed[comp], sizeof(Seed) * (size_t)n + 16);
  if (n > 0) {
    CK(cudaMemcpyAsync(ctx->io.p, seeds, (size_t)len, cudaMemcpyHostToDevice, ctx->st));
    k_seeds_in<<<grid_for(n, 256), 256, 0, ctx->st>>>(P<uint8_t>(ctx->io), n, ctx->posb, ctx->ctgb,
                                                       P<Seed>(ctx->seed[comp]));
    LAUNCHED(1);
    CK(cudaGetLastError());
  }
  ctx->nseed[comp] = n;
  ctx->have_seeds = true;
  ctx->seeds_released = false;
  ctx->have_diag[comp] = false;
  ctx->seeds_consumed[comp] = false;
  return PGA_OK;
}

int pga_diag_sort(pga_ctx *ctx, int comp, int *swide, int64_t *count) {
  if (!ctx || !ctx->have_seeds || !ctx->have_gdb || (comp != 0 && comp != 1)) return PGA_ERR_ARG;
  if (ctx->seeds_released) return fail(ctx, PGA_ERR_ARG, "seeds were freed for the alignment; run pga_merge again");
  CK(cudaSetDevice(ctx->device));
  int64_t maxdag = 2 * ctx->maxctg, cum = 1;
  int dbyte = 0;
  while (cum < maxdag) {
    cum *= 256;
    dbyte++;
  }
  if (dbyte > 4) return fail(ctx, PGA_ERR_LIMIT, "DBYTE %d > 4", dbyte);
  if (dbyte < 1) dbyte = 1;
  // sorted already (its seeds were consumed): the same result again
  if (!(ctx->seeds_consumed[comp] && ctx->have_diag[comp])) {
    int r = run_diag(ctx, comp, ctx->ncontig, ctx->maxctg, dbyte, ctx->ctgb);
    if (r) return r;
  }
  if (swide) *swide = 2 * dbyte + ctx->ctgb + 2;
  if (count) *count = ctx->nseed[comp];
  return PGA_OK;
}

int pga_diag_copy(pga_ctx *ctx, int comp, uint8_t *records, int64_t *panel_off) {
  if (!ctx || (comp != 0 && comp != 1) || !ctx->have_diag[comp]) return PGA_ERR_ARG;
  return copy_diag(ctx, comp, ctx->ncontig, records, panel_off);
}

int pga_gdb_set_freq(pga_ctx *ctx, const float *freq4) {
  if (!ctx || !freq4) return PGA_ERR_ARG;
  for (int q = 0; q < 4; q++) ctx->base_freq[q] = freq4[q];
  ctx->freq_set = true;
  return PGA_OK;
}

int pga_align(pga_ctx *ctx, int64_t *nalign) {
  if (!ctx || !ctx->have_seeds || !ctx->have_gdb) return PGA_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  AlignScope scope(ctx);
  stage_begin(ctx, ST_ALIGN);
  int r = run_align(ctx);
  if (r == PGA_ERR_NOMEM && release_for_align(ctx)) {
    cudaGetLastError();
    r = run_align(ctx);
  }
  if (r) return r;
  stage_end(ctx, ST_ALIGN);
  if (nalign) *nalign = ctx->nalign;
  return PGA_OK;
}

int pga_align_copy(pga_ctx *ctx, int32_t *recs9, int64_t *trace_off, uint8_t *trace) {
  if (!ctx || !ctx->have_align) return PGA_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  int r = host_alignments(ctx);
  if (r) return r;
  int64_t n = (int64_t)ctx->h_recs.size();
  for (int64_t i = 0; i < n; i++) {
    const AlnRec &a = ctx->h_recs[i];
    if (recs9) {
      int32_t *d = recs9 + 9 * i;
      d[0] = a.aread; d[1] = a.abpos; d[2] = a.aepos; d[3] = a.bread; d[4] = a.bbpos; d[5] = a.bepos;
      d[6] = a.comp; d[7] = a.diffs; d[8] = a.tlen;
    }
  }
  if (trace_off) memcpy(trace_off, ctx->h_toff.data(), sizeof(int64_t) * (n + 1));
  if (trace && !ctx->h_trace.empty()) memcpy(trace, ctx->h_trace.data(), ctx->h_trace.size());
  return PGA_OK;
}

int pga_local_alignment(pga_ctx *ctx, int64_t n, const int32_t *req8, int64_t *ntrace) {
  if (!ctx || !ctx->have_gdb || n < 0 || (n > 0 && !req8)) return PGA_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  AlignScope scope(ctx);
  ctx->have_local = false;
  for (int64_t i = 0; i < n; i++) {
    const int32_t *q = req8 + 8 * i;
    if (q[0] < 0 || q[0] >= ctx->ncontig || q[1] < 0 || q[1] >= ctx->ncontig || (q[2] != 0 && q[2] != 1))
      return fail(ctx, PGA_ERR_ARG, "request %lld: contigs or orientation out of range", (long long)i);
    const int64_t alen = ctx->clen[q[0]], blen = ctx->clen[q[1]];
    // the band's start points ((anti+k)/2, (anti-k)/2) must lie in the contigs
    bool in = q[3] <= q[4] && q[4] - q[3] <= 8000;
    for (int e = 3; e <= 4 && in; e++) {
      const int64_t x = ((int64_t)q[5] + q[e]) >> 1, y = x - q[e];
      in = x >= 0 && x <= alen && y >= 0 && y <= blen;
    }
    if (!in)
      return fail(ctx, PGA_ERR_ARG, "request %lld: band [%d,%d] at antidiagonal %d starts outside the contigs",
                  (long long)i, q[3], q[4], q[5]);
  }
  int ave_path = 0;
  int r = prepare_sequences(ctx, &ave_path);
  if (r) return r;
  AlignLaunch L{};
  r = prepare_workspace(ctx, L, ave_path);
  if (r) return r;
  ENSURE(ctx->lreq, sizeof(int32_t) * 8 * (size_t)(n + 1));
  ENSURE(ctx->lpath, sizeof(int32_t) * 7 * (size_t)(n + 1));
  ENSURE(ctx->ltoff, sizeof(int64_t) * (size_t)(n + 1));
  ENSURE(ctx->lnext, 64);
  int64_t tcap = 0;  // trace values: at most 2 per 100 A-bases + 4 per request
  for (int64_t i = 0; i < n; i++) tcap += 2 * (ctx->clen[req8[8 * i]] / 100 + 2);
  ENSURE(ctx->ltrace, sizeof(uint16_t) * (size_t)(tcap + 1));
  if (n > 0)
    CK(cudaMemcpyAsync(ctx->lreq.p, req8, sizeof(int32_t) * 8 * n, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemsetAsync(ctx->lnext.p, 0, 16, ctx->st));
  CK(cudaMemsetAsync(ctx->cell_next.p, 0, 8, ctx->st));
  L.lreq = P<int32_t>(ctx->lreq);
  L.nlreq = n;
  L.lreq_next = P<unsigned long long>(ctx->lnext);
  L.lpath = P<int32_t>(ctx->lpath);
  L.ltoff = P<int64_t>(ctx->ltoff);
  L.ltrace = P<uint16_t>(ctx->ltrace);
  L.ltrace_next = P<unsigned long long>(ctx->lnext) + 1;
  L.ltrace_cap = tcap;
  std::vector<int32_t> path(7 * (size_t)n);
  std::vector<int64_t> toff(n);
  for (int attempt = 0;; attempt++) {
    if (n > 0) {
      const int grid = (int)((L.nwarps * 32 + ALIGN_THREADS - 1) / ALIGN_THREADS);
      launch_local_batch(L, grid, ctx->st);
      LAUNCHED(1);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(path.data(), ctx->lpath.p, sizeof(int32_t) * 7 * n, cudaMemcpyDeviceToHost, ctx->st));
      CK(cudaMemcpyAsync(toff.data(), ctx->ltoff.p, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, ctx->st));
    }
    CK(cudaStreamSynchronize(ctx->st));
    int cells_full = 0;
    for (int64_t i = 0; i < n; i++)
      if (path[7 * i + 6] & aln::ALN_ERR_CELLS) cells_full = 1;
    const size_t max_cells = sizeof(aln::Pebble) * (size_t)0x7fffffff;
    if (!cells_full || attempt >= 6 || ctx->cells.cap >= max_cells) break;
    // grow the pebble pool and run again
    r = ensure(ctx, ctx->cells, std::min(2 * ctx->cells.cap, max_cells));
    if (r) return r;
    L.cell_cap = (int64_t)(ctx->cells.cap / sizeof(aln::Pebble));
    L.cells = P<aln::Pebble>(ctx->cells);
    CK(cudaMemsetAsync(ctx->lnext.p, 0, 16, ctx->st));
    CK(cudaMemsetAsync(ctx->cell_next.p, 0, 8, ctx->st));
  }
  // traces in request order
  ctx->h_lpath = path;
  ctx->h_ltoff.assign(n + 1, 0);
  int64_t tot = 0;
  for (int64_t i = 0; i < n; i++) {
    ctx->h_ltoff[i] = tot;
    tot += path[7 * i + 5];
  }
  ctx->h_ltoff[n] = tot;
  std::vector<uint16_t> pool(tcap + 1);
  if (tcap > 0)
    CK(cudaMemcpyAsync(pool.data(), ctx->ltrace.p, sizeof(uint16_t) * tcap, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->h_ltrace.assign(tot, 0);
  for (int64_t i = 0; i < n; i++)
    if (path[7 * i + 5] > 0)
      memcpy(ctx->h_ltrace.data() + ctx->h_ltoff[i], pool.data() + toff[i], sizeof(uint16_t) * path[7 * i + 5]);
  ctx->have_local = true;
  if (ntrace) *ntrace = tot;
  return PGA_OK;
}

int pga_local_alignment_copy(pga_ctx *ctx, int32_t *path7, int64_t *trace_off, uint16_t *trace) {
  if (!ctx || !ctx->have_local) return PGA_ERR_ARG;
  const size_t n = ctx->h_ltoff.size() - 1;
  if (path7 && n) memcpy(path7, ctx->h_lpath.data(), sizeof(int32_t) * 7 * n);
  if (trace_off) memcpy(trace_off, ctx->h_ltoff.data(), sizeof(int64_t) * (n + 1));
  if (trace && !ctx->h_ltrace.empty()) memcpy(trace, ctx->h_ltrace.data(), sizeof(uint16_t) * ctx->h_ltrace.size());
  return PGA_OK;
}

int pga_align_work(const pga_ctx *ctx, int64_t *work4) {
  if (!ctx || !work4) return PGA_ERR_ARG;
  for (int i = 0; i < 4; i++) work4[i] = ctx->align_work[i];
  return PGA_OK;
}

int pga_align_profile(const pga_ctx *ctx, int64_t *prof2) {
  if (!ctx || !prof2) return PGA_ERR_ARG;
  prof2[0] = ctx->align_prof[0];
  prof2[1] = ctx->align_prof[1];
  return PGA_OK;
}

int pga_align_set_build(pga_ctx *ctx, int ctas_per_sm) {
  if (!ctx || (ctas_per_sm != 0 && (ctas_per_sm < 2 || ctas_per_sm > 5))) return PGA_ERR_ARG;
  ctx->align_build = ctas_per_sm;
  return PGA_OK;
}

int pga_align_set_long_waves(pga_ctx *ctx, int waves) {
  if (!ctx || waves < -1) return PGA_ERR_ARG;
  ctx->long_waves = waves;
  return PGA_OK;
}

int pga_index_set_digit_bits(pga_ctx *ctx, int bits) {
  if (!ctx || (bits != 0 && (bits < MIN_DIGIT_BITS || bits > MAX_DIGIT_BITS))) return PGA_ERR_ARG;
  ctx->digit_bits = bits;
  return PGA_OK;
}

int pga_align_times(const pga_ctx *ctx, float *ms4) {
  if (!ctx || !ms4) return PGA_ERR_ARG;
  for (int i = 0; i < 4; i++) ms4[i] = ctx->align_ms[i];
  return PGA_OK;
}

int pga_align_set_ranges(pga_ctx *ctx, int64_t range_seeds) {
  if (!ctx || range_seeds < -1) return PGA_ERR_ARG;
  ctx->range_seeds = range_seeds;
  return PGA_OK;
}

static int align_write_1aln(pga_ctx *ctx, bool binary, const char *path, const char *program, const char *version,
                            const char *command, const char *db_name, const char *cwd, int nscaff,
                            const char *const *scaff_name, const int64_t *scaff_len, const int32_t *scaff_fctg,
                            const int64_t *contig_sbeg) {
  if (!ctx || !ctx->have_align) return PGA_ERR_ARG;
  if (nscaff > 0 && scaff_fctg && scaff_fctg[nscaff] > ctx->ncontig) return PGA_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  int hr = host_alignments(ctx);
  if (hr) return hr;
  const int64_t n = (int64_t)ctx->h_recs.size();
  std::vector<int32_t> r9(9 * (size_t)n);
  for (int64_t i = 0; i < n; i++) {
    const AlnRec &a = ctx->h_recs[i];
    int32_t *r = r9.data() + 9 * i;
    r[0] = a.aread;
    r[1] = a.abpos;
    r[2] = a.aepos;
    r[3] = a.bread;
    r[4] = a.bbpos;
    r[5] = a.bepos;
    r[6] = a.comp;
    r[7] = a.diffs;
    r[8] = a.tlen;
  }
  return (binary ? pga_write_1aln_binary : pga_write_1aln)(path, program, version, command, db_name, cwd,
                                                           aln::TSPACE, nscaff, scaff_name, scaff_len, scaff_fctg,
                                                           contig_sbeg, ctx->clen.data(), n, r9.data(),
                                                           ctx->h_toff.data(), ctx->h_trace.data());
}

int pga_align_write_1aln(pga_ctx *ctx, const char *path, const char *program, const char *version,
                         const char *command, const char *db_name, const char *cwd, int nscaff,
                         const char *const *scaff_name, const int64_t *scaff_len, const int32_t *scaff_fctg,
                         const int64_t *contig_sbeg) {
  return align_write_1aln(ctx, false, path, program, version, command, db_name, cwd, nscaff, scaff_name, scaff_len,
                          scaff_fctg, contig_sbeg);
}

int pga_align_write_1aln_binary(pga_ctx *ctx, const char *path, const char *program, const char *version,
                                const char *command, const char *db_name, const char *cwd, int nscaff,
                                const char *const *scaff_name, const int64_t *scaff_len,
                                const int32_t *scaff_fctg, const int64_t *contig_sbeg) {
  return align_write_1aln(ctx, true, path, program, version, command, db_name, cwd, nscaff, scaff_name, scaff_len,
                          scaff_fctg, contig_sbeg);
}

int pga_align_stats(const pga_ctx *ctx, int64_t *stats8) {
  if (!ctx || !stats8) return PGA_ERR_ARG;
  for (int i = 0; i < 8; i++) stats8[i] = ctx->align_stats[i];
  return PGA_OK;
}

int pga_fastga_ranges(int n, const int64_t *clen_pos, int64_t npost, const int64_t *seeds_pos, int64_t swide,
                      int nthreads, int *range_start) {
  if (n < 0 || nthreads <= 0 || swide <= 0 || npost < 0 ||
      (n > 0 && (!clen_pos || !seeds_pos || !range_start)))
    return PGA_ERR_ARG;
  if (n == 0) return PGA_OK;
  std::vector<int64_t> c(clen_pos, clen_pos + n), sd(seeds_pos, seeds_pos + n);
  std::vector<int> rs;
  fo_ranges(n, c, npost, sd, swide, nthreads, rs);
  std::copy(rs.begin(), rs.end(), range_start);
  return PGA_OK;
}

}  // extern "C"
