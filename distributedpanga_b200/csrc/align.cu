// Alignment stage on the GPU: every (anchor, partner) contig pair of a unit
// is one task; a persistent kernel gives each warp the next task (tasks come
// largest first), and the warp runs FastGA's chain driver and Local_Alignment
// for it (align_core.cuh, align_warp.cuh), then the pair's finishing step
// (finish.cuh: sort, elimination, joining) on the warp's lanes, and appends
// the surviving alignments.
//
// Reference: search_seeds / align_contigs / Local_Alignment
// (src/fastga_pipeline.c:576-1138, lib/align.c:1423-1576).
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>
#include "align.cuh"
#include "align_warp.cuh"
#include "finish.cuh"
#include "seeds.cuh"

namespace pga {

using namespace aln;

// Band info bits (k_band_info): the seed starts a band; the pair's previous
// band is the band just below.
constexpr uint16_t BI_START = 0x8000, BI_ADJ = 0x4000;

// One seed of a merged band block, staged in shared memory.
struct BlockSeed {
  int64_t anti;
  int lcp2, dgw;  // 2*lcp; low diagonal bits (+BUCK_WIDTH in stream 2) | stream << 16
};

// 64-bit exclusive running max in lane order, seeded with init.
__device__ __forceinline__ int64_t warp_excl_max64(int64_t v, int lane, int64_t init) {
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int64_t y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x = x > y ? x : y;
  }
  int64_t ex = __shfl_up_sync(FULL, x, 1);
  if (lane == 0) ex = init;
  return ex > init ? ex : init;
}

// Number of the 32 sorted values held one per lane (xo) below v (strictly,
// or not above it with `le`).
__device__ __forceinline__ int warp_count_below(int64_t xo, int64_t v, bool le) {
  int c = 0;
#pragma unroll
  for (int st = 16; st > 0; st >>= 1) {
    int64_t y = __shfl_sync(FULL, xo, c + st - 1);
    if (le ? (y <= v) : (y < v)) c += st;
  }
  int64_t y = __shfl_sync(FULL, xo, c);
  if (c < 32 && (le ? (y <= v) : (y < v))) c += 1;
  return c;
}

// A pair's seeds as its sorted keys, read by a whole warp: band scans test
// 32 keys per step, and a block's chains are found 32 merged seeds at a time
// (scan_block).  All lanes call every method with the same arguments.
struct KeySeeds {
  const U128 *k;
  int64_t n;
  SeedKeyLayout L;
  BlockSeed *sh;  // 32 slots of this warp's shared memory
  __device__ int64_t anti(int64_t i) const { return (int64_t)key_bits(k[i], L.off_anti, L.off_band - L.off_anti); }
  __device__ int64_t band(int64_t i) const { return (int64_t)key_bits(k[i], L.off_band, L.off_j - L.off_band); }
  __device__ int lcp(int64_t i) const { return (int)key_bits(k[i], 0, 6); }
  __device__ int dlow(int64_t i) const { return (int)key_bits(k[i], L.off_dlow, 6); }
  __device__ int64_t band_end(int64_t i, int64_t b) const {
    const int lane = threadIdx.x & 31;
    for (int64_t base = i; base < n; base += 32) {
      int64_t j = base + lane;
      bool stop = j < n && band(j) != b;
      unsigned msk = __ballot_sync(FULL, stop);
      if (msk) return base + __ffs(msk) - 1;
    }
    return n;
  }

  // The chains of the block [b, m) + [m, e) exactly as scan_block_scalar
  // finds them.  Per step each lane loads the next seed of both streams; a
  // seed's place in the merged order is its index plus the number of the
  // other stream's window seeds before it (stream 1 first on ties), and the
  // first 32 places form the step.  With P the running maximum of chain ends
  // (seeded with -CHAIN_BREAK), seed i opens a chain iff
  // anti_i >= P_before_i + CHAIN_BREAK, and adds
  // max(0, end_i - max(anti_i, P_before_i)) to its chain's coverage -- the
  // scalar loop's union length, since P_before_i is its chain's high end.
  template <class Sink>
  __device__ int scan_block(int64_t b, int64_t m, int64_t e, Sink &K) const {
    const int lane = threadIdx.x & 31;
    int64_t P = -CHAIN_BREAK;  // highest chain end so far
    bool open = false;         // a chain is open (the first seed always opens one)
    int64_t cov = 0, alow = 0;
    int mix = 0, dgmin = 0, dgmax = 0;
    int64_t s = b, t = m;
    while (s < m || t < e) {
      int64_t i1 = s + lane, i2 = t + lane;
      int64_t a1 = MAX_I64, a2 = MAX_I64;
      int l1 = 0, l2 = 0, d1 = 0, d2 = 0;
      if (i1 < m) {
        U128 key = k[i1];
        a1 = (int64_t)key_bits(key, L.off_anti, L.off_band - L.off_anti);
        l1 = (int)key_bits(key, 0, 6);
        d1 = (int)key_bits(key, L.off_dlow, 6);
      }
      if (i2 < e) {
        U128 key = k[i2];
        a2 = (int64_t)key_bits(key, L.off_anti, L.off_band - L.off_anti);
        l2 = (int)key_bits(key, 0, 6);
        d2 = (int)key_bits(key, L.off_dlow, 6);
      }
      int take1, take2;
      int64_t anti;
      int lcp2, dg, wch;
      int cnt;
      if (t >= e) {
        // stream 1 alone
        take1 = (m - s) < 32 ? (int)(m - s) : 32;
        take2 = 0;
        cnt = take1;
        anti = a1;
        lcp2 = l1 << 1;
        dg = d1;
        wch = 1;
      } else {
        int r1 = lane + warp_count_below(a2, a1, false);
        int r2 = lane + warp_count_below(a1, a2, true);
        bool g1 = i1 < m && r1 < 32, g2 = i2 < e && r2 < 32;
        take1 = __popc(__ballot_sync(FULL, g1));
        take2 = __popc(__ballot_sync(FULL, g2));
        cnt = take1 + take2;
        if (g1) sh[r1] = BlockSeed{a1, l1 << 1, d1 | (1 << 16)};
        if (g2) sh[r2] = BlockSeed{a2, l2 << 1, (d2 + BUCK_WIDTH) | (2 << 16)};
        __syncwarp();
        BlockSeed q = sh[lane];
        __syncwarp();
        anti = q.anti;
        lcp2 = q.lcp2;
        dg = q.dgw & 0xffff;
        wch = q.dgw >> 16;
      }
      const bool valid = lane < cnt;
      const int64_t end = valid ? anti + lcp2 : -MAX_I64;
      const int64_t pb = warp_excl_max64(end, lane, P);  // P before this seed
      const bool brk = valid && anti >= pb + CHAIN_BREAK;
      int64_t hi = pb > anti ? pb : anti;
      const int add = valid ? (end > hi ? (int)(end - hi) : 0) : 0;
      uint32_t bm = __ballot_sync(FULL, brk);
      int lo = 0;
      while (true) {
        // seeds [lo, stop) continue the open chain
        int stop = bm ? __ffs(bm) - 1 : cnt;
        if (stop > lo) {
          bool in = lane >= lo && lane < stop;
          cov += __reduce_add_sync(FULL, in ? add : 0);
          mix |= (int)__reduce_or_sync(FULL, in ? (unsigned)wch : 0u);
          dgmin = min(dgmin, __reduce_min_sync(FULL, in ? dg : 2147483647));
          dgmax = max(dgmax, __reduce_max_sync(FULL, in ? dg : -2147483647));
        }
        if (!bm) break;
        // seed `stop` ends the open chain and opens the next
        const int64_t ahgh = __shfl_sync(FULL, pb, stop);
        if (open && K.chain(cov, mix, dgmin, dgmax, alow, ahgh)) return 1;
        open = true;
        cov = __shfl_sync(FULL, add, stop);
        mix = __shfl_sync(FULL, wch, stop);
        dgmin = dgmax = __shfl_sync(FULL, dg, stop);
        alow = __shfl_sync(FULL, anti, stop);
        lo = stop + 1;
        bm &= bm - 1;
      }
      int64_t em = end;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        int64_t y = __shfl_xor_sync(FULL, em, o);
        em = em > y ? em : y;
      }
      if (em > P) P = em;
      s += take1;
      t += take2;
    }
    if (open) return K.chain(cov, mix, dgmin, dgmax, alow, P);
    return 0;
  }
};

struct WarpAligner {
  WarpWork &W;
  const AlignSpec &spec;
  const CallMemo &M;
  int a, b;  // the pair's contigs (A's and B's)
  __device__ int call(const Seq &A, const Seq &B, bool acomp, Path &P, int low, int hgh, int anti, int lbord,
                      int hbord) {
    const long long t0 = clock64();
    const int lane = threadIdx.x & 31;
    // a call on two target contigs: its recorded result, if the target's run made it
    const bool keyed = (M.cap > 0 || M.lkey) && a < M.nt && b < M.nt;
    uint32_t k[MEMO_KEY];
    k[0] = (uint32_t)a | ((uint32_t)b << 15) | ((uint32_t)acomp << 30);
    k[1] = (uint32_t)low;
    k[2] = (uint32_t)hgh;
    k[3] = (uint32_t)anti;
    k[4] = (uint32_t)lbord;
    k[5] = (uint32_t)hbord;
    if (keyed && M.cap > 0) {
      const uint64_t mask = (uint64_t)M.cap - 1;
      for (uint64_t s = memo_hash(k) & mask, probe = 0; probe <= mask; probe++, s = (s + 1) & mask) {
        const uint32_t *q = M.key + MEMO_KEY * s;
        if (q[0] == MEMO_EMPTY) break;
        bool same = true;
        for (int i = 0; i < MEMO_KEY; i++) same &= q[i] == k[i];
        if (!same) continue;
        const int32_t *v = M.val + MEMO_VAL * s;
        if (v[5] > W.point_cap) break;  // computed below, which reports the overflow
        const uint8_t *tr = M.trace + M.toff[s];
        for (int i = lane; i < v[5]; i += 32) W.points[i] = tr[i];
        __syncwarp();
        P.abpos = v[0];
        P.aepos = v[1];
        P.bbpos = v[2];
        P.bepos = v[3];
        P.diffs = v[4];
        P.tlen = v[5];
        P.trace_off = 0;
        if (lane == 0) atomicAdd(M.hits, 1ull);
        W.la_cycles += clock64() - t0;
        return 0;
      }
    }
    const int r = local_alignment_w(W, spec, A, B, acomp, P, low, hgh, anti, lbord, hbord);
    if (keyed && M.lkey && r == 0) {
      // the target's own run: append the call to the log
      unsigned long long e = 0, tb = 0;
      if (lane == 0) {
        e = atomicAdd(M.lnext, 1ull);
        tb = atomicAdd(M.lbytes, (unsigned long long)P.tlen);
      }
      e = __shfl_sync(FULL, e, 0);
      tb = __shfl_sync(FULL, tb, 0);
      if ((int64_t)e < M.lcap) {
        const bool fits = (int64_t)(tb + P.tlen) <= M.lbytes_cap;
        if (fits)
          for (int i = lane; i < P.tlen; i += 32) M.ltrace[tb + i] = (uint8_t)W.points[P.trace_off + i];
        if (lane == 0) {
          for (int i = 0; i < MEMO_KEY; i++) M.lkey[MEMO_KEY * e + i] = k[i];
          int32_t *v = M.lval + MEMO_VAL * e;
          v[0] = P.abpos;
          v[1] = P.aepos;
          v[2] = P.bbpos;
          v[3] = P.bepos;
          v[4] = P.diffs;
          v[5] = P.tlen;
          M.ltoff[e] = fits ? (int64_t)tb : -1;
        }
      }
      __syncwarp();
    }
    W.la_cycles += clock64() - t0;
    return r;
  }
  __device__ const uint16_t *points() const { return W.points; }
  __device__ int err() const { return W.err; }
};

__device__ AlignSpec launch_spec(const AlignLaunch &P) {
  AlignSpec spec;
  spec.trace_space = TSPACE;
  spec.ave_path = P.ave_path;
  spec.reach = 0;
  spec.score = P.score;
  spec.table = P.table;
  return spec;
}

// Warp wid's wave buffers, trace points and pebble pool.
__device__ WarpWork warp_work(const AlignLaunch &P, int64_t wid) {
  WarpWork W;
  int *wb = P.wave + wid * (int64_t)P.vcap * WAVE_INTS;
  W.V[0] = wb;
  W.V[1] = wb + P.vcap;
  W.M[0] = wb + 2 * P.vcap;
  W.M[1] = wb + 3 * P.vcap;
  W.HA[0] = wb + 4 * P.vcap;
  W.HA[1] = wb + 5 * P.vcap;
  W.NA = wb + 6 * P.vcap;
  W.HM[0] = wb + 7 * P.vcap;
  W.HM[1] = wb + 8 * P.vcap;
  W.T[0] = (uint64_t *)(wb + 9 * P.vcap);
  W.T[1] = (uint64_t *)(wb + 11 * P.vcap);
  W.vcap = P.vcap;
  W.points = P.points + wid * P.point_cap;
  W.point_cap = P.point_cap;
  W.pool.cells = P.cells;
  W.pool.next = P.cell_next;
  W.pool.cap = P.cell_cap;
  W.chunk_next = W.chunk_end = 0;
  W.waves = W.cells = 0;
  W.smflag = P.smflag;
  W.long_waves = P.smflag ? P.long_waves : 0;
  W.flagged = 0;
  W.la_cycles = 0;
  return W;
}

// Sequences of contig c as a Local_Alignment operand: A is complemented
// when comp (the reverse-complement copies), B never.
__device__ Seq contig_seq(const AlignLaunch &P, int c, bool as_a, bool comp) {
  const uint8_t *buf = (as_a && comp) ? P.rc : P.fwd;
  Seq S{buf + P.soff[c], (int)P.clen[c]};
  const uint64_t *base = P.pk + P.poff[c] * 4;
  if (as_a) {
    S.pf = base + (comp ? 2 : 0) * P.pwords[c];
    S.pr = base + (comp ? 3 : 1) * P.pwords[c];
  } else {
    S.pf = base;
    S.pr = base + P.pwords[c];
  }
  return S;
}

__device__ OvlArena warp_arena(const AlignLaunch &P, int64_t wid) {
  OvlArena O;
  O.ovl = P.ovl + wid * P.ovl_cap;
  O.perm = P.perm + wid * 2 * P.ovl_cap;
  O.tmp = O.perm + P.ovl_cap;
  O.ovl_cap = P.ovl_cap;
  O.bytes = P.cand_bytes;
  O.pool_next = P.cand_next;
  O.pool_cap = P.cand_cap;
  O.nbyte = O.byte_cap = 0;
  O.nov = 0;
  O.err = 0;
  return O;
}

// First index >= x in [x, hi) whose band differs from its predecessor's
// (x itself when x == 0), else hi; warp-wide.  Bands never decrease within
// a pair, so this is the first index whose band exceeds band(x-1): a search
// that probes 32 points per step (ballot) and ends with one linear step of
// 32, so a range that starts inside a long band does not walk its seeds.
__device__ int64_t next_band_start(const KeySeeds &S, int64_t x, int64_t hi, int lane) {
  if (x <= 0) return 0;
  if (x >= hi) return hi;
  const int64_t b = S.band(x - 1);
  int64_t lo = x, h = hi;  // the answer lies in [lo, h], h meaning none below h
  while (h - lo > 32) {
    const int64_t span = h - lo;
    const int64_t p = lo + (span * (lane + 1)) / 33;  // increasing in lane, inside [lo, h)
    const unsigned m = __ballot_sync(FULL, S.band(p) > b);
    if (m) {
      const int f = __ffs(m) - 1;
      const int64_t pf = lo + (span * (f + 1)) / 33;
      const int64_t before = f > 0 ? lo + (span * f) / 33 : lo - 1;  // last probe known not past b
      lo = before + 1;
      h = pf;  // band(pf) > b: the answer is at most pf
      if (h - lo <= 32) {
        const int64_t q = lo + lane;
        const unsigned m2 = __ballot_sync(FULL, q < h && S.band(q) > b);
        return m2 ? lo + __ffs(m2) - 1 : h;
      }
    } else {
      lo = lo + (span * 32) / 33 + 1;
    }
  }
  const int64_t q = lo + lane;
  const unsigned m = __ballot_sync(FULL, q < h && S.band(q) > b);
  return m ? lo + __ffs(m) - 1 : h;
}

// align_pair (align_core.cuh) for a pair's seeds on the device: the same
// band blocks in the same order, with the same chains and calls, but the
// blocks come from the per-seed band info, 32 seeds per step, and a block
// whose seeds' 2*lcp sum is below CHAIN_MIN is passed over: a chain's
// coverage is at most the sum of its seeds' spans, so no chain of it can
// pass the hit test, and such a block makes no call and changes no state.
// Block (c, c+1) starting at band c's first seed b is scanned when band c
// is new (the band below it is not c-1) or band c+1 follows it, as in
// align_pair; blocks start in [blo, bhi).
template <class Aligner>
__device__ int align_pair_dev(const KeySeeds &S, const uint16_t *info, bool comp, bool self, const Seq &A,
                              const Seq &B, int64_t amxpos, int64_t maxdag, Aligner &AL, Path &path, OvlArena &O,
                              PairResult &R, int lane, int64_t blo, int64_t bhi) {
  const int64_t n = S.n;
  R.calls = 0;
  R.nhit = 0;
  R.nlas = 0;
  R.exit_bepos = path.bepos;
  O.nov = 0;
  if (bhi < 0 || bhi > n) bhi = n;
  if (blo < 0) blo = 0;
  if (blo >= bhi) return 0;
  ChainSink<WarpAligner> K{comp, self, A, B, AL, path, O, R, lane, 32, amxpos, (int64_t)A.len + B.len,
                           (int64_t)A.len - maxdag, (int64_t)A.len - amxpos, 0, 0, -1};
  int64_t pend = -1;  // the last band start seen, its block not yet decided
  int pend_sum = 0;
  bool pend_new = false;
  bool done = false;
  for (int64_t base = blo; base < n && !done; base += 32) {
    const int64_t i = base + lane;
    const uint16_t v = i < n ? info[i] : 0;
    unsigned starts = __ballot_sync(FULL, (v & BI_START) != 0);
    while (starts) {
      const int l = __ffs(starts) - 1;
      starts &= starts - 1;
      const int64_t b = base + l;
      const uint16_t vb = __shfl_sync(FULL, v, l);
      if (pend >= 0) {
        const bool aux = (vb & BI_ADJ) != 0;  // band c+1 follows band c
        if ((pend_new || aux) && pend_sum + (aux ? (vb & 0xff) : 0) >= CHAIN_MIN) {
          const int64_t e = aux ? S.band_end(b, S.band(b)) : b;
          K.cdiag = S.band(pend);
          K.isnew = pend_new ? 1 : 0;
          K.alast = -1;
          if (S.scan_block(pend, b, e, K)) return 1;
        }
        pend = -1;
      }
      if (b >= bhi) {
        done = true;
        break;
      }
      pend = b;
      pend_sum = vb & 0xff;
      pend_new = (vb & BI_ADJ) == 0;
    }
  }
  if (pend >= 0 && pend_new && pend_sum >= CHAIN_MIN) {  // the pair's last band: no band after it
    K.cdiag = S.band(pend);
    K.isnew = 1;
    K.alast = -1;
    if (S.scan_block(pend, n, n, K)) return 1;
  }
  R.exit_bepos = path.bepos;
  return 0;
}

// The sort / elimination step of a pair whose candidates are in O, then its
// survivors appended to the output in the pair's order (lane 0 ranks them).
__device__ void finish_and_emit(const AlignLaunch &P, OvlArena &O, int a, int b, int comp, PairOut &po,
                                int lane) {
  const long long t0 = clock64();
  finish_candidates(Lanes{}, O);  // every lane, with the same O
  if (lane == 0 && O.nov > 0) atomicAdd(&P.prof[1], (unsigned long long)(clock64() - t0));
  if (O.err) {
    po.err = O.err | 0x200;
    return;
  }
  int ns = 0;
  int64_t tb = 0;
  if (lane == 0)
    for (int64_t q = 0; q < O.nov; q++) {
      const Ovl &o = O.ovl[O.perm[q]];
      if (o.flags & ELIMINATED) continue;
      ns++;
      tb += o.tlen;
    }
  ns = __shfl_sync(FULL, ns, 0);
  tb = __shfl_sync(FULL, tb, 0);
  unsigned long long r0 = 0, b0 = 0;
  if (lane == 0 && ns > 0) {
    r0 = atomicAdd(P.rec_next, (unsigned long long)ns);
    b0 = atomicAdd(P.out_next, (unsigned long long)tb);
  }
  r0 = __shfl_sync(FULL, r0, 0);
  b0 = __shfl_sync(FULL, b0, 0);
  if (ns > 0 && ((int64_t)(r0 + ns) > P.rec_cap || (int64_t)(b0 + tb) > P.out_cap)) {
    po.err = ALN_ERR_OVLS | 0x400;
    return;
  }
  if (ns == 0) return;
  int64_t rr = (int64_t)r0, bb = (int64_t)b0;
  int rank = 0;
  for (int64_t q = 0; q < O.nov; q++) {
    const Ovl o = O.ovl[O.perm[q]];
    if (o.flags & ELIMINATED) continue;
    if (lane == 0) {
      AlnRec &r = P.recs[rr];
      r.aread = a;
      r.bread = b;
      r.comp = comp;
      r.abpos = o.abpos;
      r.aepos = o.aepos;
      r.bbpos = o.bbpos;
      r.bepos = o.bepos;
      r.diffs = o.diffs;
      r.tlen = o.tlen;
      r.rank = rank;
      r.toff = bb;
    }
    for (int q2 = lane; q2 < o.tlen; q2 += 32) P.out_bytes[bb + q2] = P.cand_bytes[o.toff + q2];
    rr++;
    bb += o.tlen;
    rank++;
  }
  po.nsurv = ns;
  po.rec_off = (int64_t)r0;
}

__device__ __forceinline__ PairTask small_task(const AlignLaunch &P, uint64_t code) {
  const int u = (int)(code >> 63);
  const int64_t p = (int64_t)(code & 0x7fffffffffffffffull);
  PairTask t;
  t.comp = u;
  t.a = P.pab[u][2 * p];
  t.b = P.pab[u][2 * p + 1];
  t.self = 0;
  t.entry_bepos = 0;
  t.seg = -1;
  t.lo = P.pstart[u][p];
  t.hi = p + 1 < P.npairs[u] ? P.pstart[u][p + 1] : P.nseeds[u];
  t.slo = t.lo;
  t.shi = t.hi;
  return t;
}

// A warp's running reduction of its device-planned pairs' outcomes (lane 0).
struct SmallSums {
  unsigned long long calls = 0, cycles = 0, maxkey = 0, err = 0, waves = 0, cells = 0, bad = ~0ull;
  __device__ void add(const AlignLaunch &P, const PairTask &tk, const PairOut &po, unsigned t) {
    calls += (unsigned long long)po.calls;
    cycles += (unsigned long long)po.cycles;
    const unsigned long long k = ((unsigned long long)po.cycles << 16) | (unsigned)min(po.calls, 65535);
    maxkey = k > maxkey ? k : maxkey;
    if (po.err) {
      err |= (unsigned long long)po.err;
      bad = t < bad ? t : bad;
    }
    waves += (unsigned long long)po.waves;
    cells += (unsigned long long)po.cells;
    if (tk.comp == 0 && po.calls > 0) {
      const int xa = P.fo_pos[tk.a], xb = P.fo_pos[tk.b];
      const unsigned long long key = ((unsigned long long)(xb + 1) << 32) | (uint32_t)po.exit_bepos;
      atomicMax(&P.fo_last[xa], key);
      if (xb < xa) atomicMax(&P.fo_earlier[xa], key);
    }
  }
  __device__ void flush(const AlignLaunch &P) {
    if (calls) atomicAdd(&P.sred[0], calls);
    if (cycles) atomicAdd(&P.sred[1], cycles);
    if (maxkey) atomicMax(&P.sred[2], maxkey);
    if (err) atomicOr(&P.sred[3], err);
    if (waves) atomicAdd(&P.sred[4], waves);
    if (cells) atomicAdd(&P.sred[5], cells);
    if (bad != ~0ull) atomicMin(&P.sred[6], bad);
  }
};

// The persistent alignment loop, in four builds: MINB = 1 keeps every
// register a warp's wave loop wants (255, two CTAs per SM), for launches
// bounded by their longest task; MINB = 3, 4 and 5 trade spills for more
// resident warps (three to five CTAs per SM: 168, 128 or 96 registers), for
// launches bounded by throughput (many pairs), where a wave step's latency
// is hidden by the other warps of its SM (five: the 2 x 1 Gbp pair launch
// 3.50 s against 3.70 with four).
template <int MINB>
__global__ void __launch_bounds__(ALIGN_THREADS, MINB) k_align_pairs(AlignLaunch P) {
  __shared__ BlockSeed s_block[ALIGN_THREADS / 32][32];
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * ALIGN_THREADS + threadIdx.x) >> 5;
  if (wid >= P.nwarps) return;
  const AlignSpec spec = launch_spec(P);
  WarpWork W = warp_work(P, wid);

  OvlArena O = warp_arena(P, wid);
  SmallSums sums;

  while (true) {
    unsigned t = 0;
    if (W.long_waves > 0 && !W.flagged) {
      // another warp of this SM runs a long call: leave the SM to it (the
      // queue is drained by the other SMs' warps, and by the flagging warps)
      unsigned sm, f = 0;
      asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
      if (lane == 0 && sm < SM_FLAGS) f = *(volatile unsigned *)&P.smflag[sm];
      f = __shfl_sync(FULL, f, 0);
      if (f) break;
    }
    if (lane == 0) t = atomicAdd(P.next_task, 1u);
    t = __shfl_sync(FULL, t, 0);
    if (t >= (unsigned)P.ntasks + (unsigned)P.nsmall) break;
    const PairTask tk = t < (unsigned)P.ntasks ? P.tasks[t] : small_task(P, P.small[t - P.ntasks]);
    W.err = 0;
    O.err = 0;
    const SeedKeyLayout &L = tk.comp ? P.layC : P.layN;
    KeySeeds S{(tk.comp ? P.keysC : P.keysN) + tk.lo, tk.hi - tk.lo, L, s_block[threadIdx.x >> 5]};
    const Seq A = contig_seq(P, tk.a, true, tk.comp != 0);
    const Seq B = contig_seq(P, tk.b, false, false);
    long long t0 = clock64();
    Path path;
    path.tlen = path.diffs = path.abpos = path.bbpos = path.aepos = 0;
    path.bepos = tk.entry_bepos;
    path.trace_off = 0;
    int64_t blo = 0, bhi = S.n;
    if (tk.seg >= 0) {
      blo = next_band_start(S, tk.slo - tk.lo, S.n, lane);
      bhi = next_band_start(S, tk.shi - tk.lo, S.n, lane);
    }
    PairResult R;
    WarpAligner AL{W, spec, P.memo, tk.a, tk.b};
    const uint16_t *info = (tk.comp ? P.infoC : P.infoN) + tk.lo;
    int rc = align_pair_dev(S, info, tk.comp != 0, tk.self != 0, A, B, P.amxpos, P.maxdag, AL, path, O, R, lane,
                            blo, bhi);
    __syncwarp();
    PairOut po;
    po.waves = W.waves;
    po.cells = W.cells;
    W.waves = W.cells = 0;
    po.calls = R.calls;
    po.exit_bepos = R.exit_bepos;
    po.nsurv = 0;
    po.rec_off = 0;
    po.err = rc ? (W.err | O.err | 0x100) : 0;
    if (rc == 0 && tk.seg >= 0) {
      // a band range: its candidates to the range store, in order
      unsigned long long g0 = 0;
      if (lane == 0 && O.nov > 0) g0 = atomicAdd(P.rng_next, (unsigned long long)O.nov);
      g0 = __shfl_sync(FULL, g0, 0);
      if ((int64_t)g0 + O.nov > P.rng_cap) {
        po.err = ALN_ERR_OVLS | 0x800;
      } else {
        for (int64_t q = lane; q < O.nov; q += 32) P.rng_ovl[g0 + q] = O.ovl[q];
        po.nsurv = (int)O.nov;
        po.rec_off = (int64_t)g0;
      }
    }
    po.cycles = clock64() - t0;
    if (tk.seg >= 0) {
      if (lane == 0) P.rout[tk.seg] = po;
    } else if (rc == 0) {
      finish_and_emit(P, O, tk.a, tk.b, tk.comp, po, lane);
      po.cycles = clock64() - t0;
    }
    if (lane == 0) {
      if (t < (unsigned)P.ntasks) P.pout[t] = po;
      else sums.add(P, tk, po, t);
    }
    __syncwarp();
  }
  if (lane == 0 && P.nsmall > 0) sums.flush(P);
  if (lane == 0 && W.la_cycles > 0) atomicAdd(&P.prof[0], (unsigned long long)W.la_cycles);
}


// Finishes the pairs that ran as band ranges: gathers each pair's candidates
// from its ranges in range order (the order one warp running the whole pair
// would have made them in), then the pair's sort / elimination step and
// output.  The pair's calls are the ranges' sum and its exit bepos the last
// range's with a call (the entry value when none called).
__global__ void __launch_bounds__(ALIGN_THREADS)
k_finish_pairs(AlignLaunch P) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * ALIGN_THREADS + threadIdx.x) >> 5;
  if (wid >= P.nwarps) return;
  OvlArena O = warp_arena(P, wid);
  for (int64_t t = wid; t < P.nftasks; t += P.nwarps) {
    const FinishTask ft = P.ftasks[t];
    long long t0 = clock64();
    PairOut po;
    po.waves = po.cells = 0;
    po.calls = 0;
    po.exit_bepos = ft.entry_bepos;
    po.nsurv = 0;
    po.rec_off = 0;
    po.err = 0;
    O.nov = 0;
    O.err = 0;
    for (int k = 0; k < ft.nseg; k++) {
      const PairOut ro = P.rout[P.range_idx[ft.first + k]];
      po.calls += ro.calls;
      if (ro.calls > 0) po.exit_bepos = ro.exit_bepos;
      if (O.nov + ro.nsurv > O.ovl_cap) {
        po.err = ALN_ERR_OVLS | 0x1000;
        break;
      }
      for (int q = lane; q < ro.nsurv; q += 32) O.ovl[O.nov + q] = P.rng_ovl[ro.rec_off + q];
      O.nov += ro.nsurv;
    }
    __syncwarp();
    if (po.err == 0) finish_and_emit(P, O, ft.a, ft.b, ft.comp, po, lane);
    po.cycles = clock64() - t0;
    if (lane == 0) P.pout[t] = po;
    __syncwarp();
  }
}

// Local_Alignment on request lists (pga_local_alignment): warps take
// requests in turn (a b comp low hgh anti lbord hbord); each writes its path
// (abpos aepos bbpos bepos diffs tlen status) and copies its tlen uint16
// trace values into a shared pool.
__global__ void __launch_bounds__(ALIGN_THREADS)
k_local_batch(AlignLaunch P) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * ALIGN_THREADS + threadIdx.x) >> 5;
  if (wid >= P.nwarps) return;
  const AlignSpec spec = launch_spec(P);
  WarpWork W = warp_work(P, wid);
  while (true) {
    unsigned long long r = 0;
    if (lane == 0) r = atomicAdd(P.lreq_next, 1ull);
    r = __shfl_sync(FULL, r, 0);
    if ((int64_t)r >= P.nlreq) break;
    const int32_t *q = P.lreq + 8 * r;
    const bool comp = q[2] != 0;
    const Seq A = contig_seq(P, q[0], true, comp);
    const Seq B = contig_seq(P, q[1], false, false);
    W.err = 0;
    Path path;
    path.tlen = path.diffs = path.abpos = path.bbpos = path.aepos = path.bepos = 0;
    path.trace_off = 0;
    int status = local_alignment_w(W, spec, A, B, comp, path, q[3], q[4], q[5], q[6], q[7]) ? (W.err | 0x100) : 0;
    int64_t off = -1;
    if (status == 0 && path.tlen > 0) {
      unsigned long long o = 0;
      if (lane == 0) o = atomicAdd(P.ltrace_next, (unsigned long long)path.tlen);
      o = __shfl_sync(FULL, o, 0);
      if ((int64_t)o + path.tlen > P.ltrace_cap) {
        status = ALN_ERR_TRACE | 0x200;
      } else {
        off = (int64_t)o;
        for (int k = lane; k < path.tlen; k += 32) P.ltrace[off + k] = W.points[path.trace_off + k];
      }
    }
    if (lane == 0) {
      int32_t *o7 = P.lpath + 7 * r;
      o7[0] = path.abpos;
      o7[1] = path.aepos;
      o7[2] = path.bbpos;
      o7[3] = path.bepos;
      o7[4] = path.diffs;
      o7[5] = status ? 0 : path.tlen;
      o7[6] = status;
      P.ltoff[r] = off;
    }
    __syncwarp();
  }
}

void launch_local_batch(const AlignLaunch &P, int grid, cudaStream_t st) {
  k_local_batch<<<grid, ALIGN_THREADS, 0, st>>>(P);
}

// NUMERIC copies of every contig, each between sentinel bytes (value 4):
// fwd holds the contig, rc its reverse complement (Complement_Seq,
// lib/align.c:4082), both starting at soff[c].
__global__ void k_numeric(const uint8_t *__restrict__ bps, const int64_t *__restrict__ clen,
                          const int64_t *__restrict__ boff, const int64_t *__restrict__ soff, int ncontig,
                          uint8_t *__restrict__ fwd, uint8_t *__restrict__ rc) {
  int c = blockIdx.y;
  if (c >= ncontig) return;
  int64_t n = clen[c], o = soff[c];
  const uint8_t *cb = bps + boff[c];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint8_t b = (cb[i >> 2] >> (2 * (i & 3))) & 3;
    fwd[o + i] = b;
    rc[o + (n - 1 - i)] = 3 - b;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    fwd[o - 1] = fwd[o + n] = 4;
    rc[o - 1] = rc[o + n] = 4;
  }
}

// 2-bit packed copies of every contig, 32 bases per word, first base in the
// top bits, one zero pad word after each: forward, reversed, reverse
// complement and complement-only (the reverse of the reverse complement) --
// the packed forms of the sequences the forward and reverse snakes read.
__global__ void k_pack(const uint8_t *__restrict__ fwd, const int64_t *__restrict__ soff,
                       const int64_t *__restrict__ clen, const int64_t *__restrict__ poff,
                       const int64_t *__restrict__ pwords, int ncontig, uint64_t *__restrict__ pk) {
  int c = blockIdx.y;
  if (c >= ncontig) return;
  int64_t n = clen[c], nw = pwords[c];
  const uint8_t *s = fwd + soff[c];
  uint64_t *F = pk + poff[c] * 4, *R = F + nw, *RC = F + 2 * nw, *CO = F + 3 * nw;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (int64_t)gridDim.x * blockDim.x) {
    uint64_t f = 0, r = 0, rc = 0, co = 0;
    for (int q = 0; q < 32; q++) {
      int64_t i = 32 * w + q;
      uint64_t bf = 0, br = 0;
      if (i < n) {
        bf = s[i];
        br = s[n - 1 - i];
      }
      f |= bf << (62 - 2 * q);
      r |= br << (62 - 2 * q);
      rc |= (i < n ? (3 - br) : 0) << (62 - 2 * q);
      co |= (i < n ? (3 - bf) : 0) << (62 - 2 * q);
    }
    F[w] = f;
    R[w] = r;
    RC[w] = rc;
    CO[w] = co;
  }
}

void launch_pack(const uint8_t *fwd, const int64_t *soff, const int64_t *clen, const int64_t *poff,
                 const int64_t *pwords, int ncontig, uint64_t *pk, cudaStream_t st) {
  if (ncontig <= 0) return;
  dim3 g(64, ncontig);
  k_pack<<<g, 256, 0, st>>>(fwd, soff, clen, poff, pwords, ncontig, pk);
}

// Pair boundaries of a sorted key array: flag[i] = 1 where (icont, jcont)
// differs from key i-1.
// Per seed of a unit's sorted keys: whether it starts a band (its (anchor,
// partner, band) differs from the previous seed's), whether the previous
// band of the same pair is the band just below (the block before reaches it
// as its second stream), and at a band start the sum of 2*lcp over the
// band's seeds capped at CHAIN_MIN.  A band start walks at most CHAIN_MIN / 2
// seeds: every seed adds at least 2, so that many reach the cap.
__global__ void k_band_info(const U128 *__restrict__ keys, int64_t n, SeedKeyLayout L, uint16_t *__restrict__ info) {
  const int wb = L.off_j - L.off_band;                  // band field width
  const int wk = L.total_bits - L.off_band;             // band + partner + anchor
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t me = key_bits(keys[i], L.off_band, wk);
    const uint64_t prev = i > 0 ? key_bits(keys[i - 1], L.off_band, wk) : ~0ull;
    if (i > 0 && prev == me) {
      info[i] = 0;
      continue;
    }
    const uint64_t bmask = (1ull << wb) - 1;
    const bool adj = i > 0 && (prev >> wb) == (me >> wb) && (prev & bmask) + 1 == (me & bmask);
    int sum = 0;
    for (int64_t j = i; j < n && sum < CHAIN_MIN; j++) {
      const U128 k = keys[j];
      if (key_bits(k, L.off_band, wk) != me) break;
      sum += (int)key_bits(k, 0, 6) << 1;
    }
    info[i] = BI_START | (adj ? BI_ADJ : 0) | (uint16_t)(sum < CHAIN_MIN ? sum : CHAIN_MIN);
  }
}

__global__ void k_pair_flags(const U128 *__restrict__ keys, int64_t n, SeedKeyLayout L, uint32_t *__restrict__ flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t f = 1;
    if (i > 0) {
      uint64_t a = key_bits(keys[i], L.off_j, L.w_i + (L.off_i - L.off_j));
      uint64_t b = key_bits(keys[i - 1], L.off_j, L.w_i + (L.off_i - L.off_j));
      f = a != b;
    }
    flag[i] = f;
  }
}

// Compact the pair starts: pos[idx[i]] = i where flag[i]; also the pair's
// anchor and partner.
__global__ void k_pair_starts(const U128 *__restrict__ keys, int64_t n, SeedKeyLayout L,
                              const uint32_t *__restrict__ flag, const uint32_t *__restrict__ idx,
                              int64_t *__restrict__ start, int32_t *__restrict__ ab) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    uint32_t p = idx[i];
    start[p] = i;
    ab[2 * p] = (int32_t)key_bits(keys[i], L.off_i, L.w_i);
    ab[2 * p + 1] = (int32_t)key_bits(keys[i], L.off_j, L.off_i - L.off_j);
  }
}

// Base counts (A, C, G, T) over all contigs with sequence.
__global__ void k_base_counts(const uint8_t *__restrict__ bps, const int64_t *__restrict__ clen,
                              const int64_t *__restrict__ boff, int ncontig, unsigned long long *__restrict__ cnt) {
  __shared__ unsigned long long sc[4];
  if (threadIdx.x < 4) sc[threadIdx.x] = 0;
  __syncthreads();
  int c = blockIdx.y;
  unsigned long long l[4] = {0, 0, 0, 0};
  if (c < ncontig && boff[c] >= 0) {
    int64_t n = clen[c];
    const uint8_t *cb = bps + boff[c];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      l[(cb[i >> 2] >> (2 * (i & 3))) & 3]++;
  }
  for (int q = 0; q < 4; q++) {
    unsigned long long v = l[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&sc[q], v);
  }
  __syncthreads();
  if (threadIdx.x < 4) atomicAdd(&cnt[threadIdx.x], sc[threadIdx.x]);
}

void launch_base_counts(const uint8_t *bps, const int64_t *clen, const int64_t *boff, int ncontig,
                        unsigned long long *cnt, cudaStream_t st) {
  if (ncontig <= 0) return;
  dim3 g(16, ncontig);
  k_base_counts<<<g, 256, 0, st>>>(bps, clen, boff, ncontig, cnt);
}

void launch_align(const AlignLaunch &P, int grid, cudaStream_t st) {
  if (P.min_blocks == 5) k_align_pairs<5><<<grid, ALIGN_THREADS, 0, st>>>(P);
  else if (P.min_blocks == 4) k_align_pairs<4><<<grid, ALIGN_THREADS, 0, st>>>(P);
  else if (P.min_blocks == 3) k_align_pairs<3><<<grid, ALIGN_THREADS, 0, st>>>(P);
  else k_align_pairs<1><<<grid, ALIGN_THREADS, 0, st>>>(P);
}

void launch_finish(const AlignLaunch &P, int grid, cudaStream_t st) {
  k_finish_pairs<<<grid, ALIGN_THREADS, 0, st>>>(P);
}

// For each self pair [lo, hi) of the N unit: the first seed whose band is
// >= cd_lo and the first whose band is > cd_hi (relative to lo).  The band
// blocks between are the only ones whose diagonal span can hold diagonal 0.
__global__ void k_self_bounds(const U128 *__restrict__ keys, SeedKeyLayout L, const int64_t *__restrict__ lohi,
                              int npair, int64_t cd_lo, int64_t cd_hi, int64_t *__restrict__ x12) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npair) return;
  const int64_t lo = lohi[2 * q], hi = lohi[2 * q + 1];
  for (int w = 0; w < 2; w++) {
    // first index in [lo, hi) with band > lim (lim = cd_lo - 1, then cd_hi)
    const int64_t lim = w == 0 ? cd_lo - 1 : cd_hi;
    int64_t a = lo, b = hi;
    while (a < b) {
      int64_t mid = a + (b - a) / 2;
      int64_t band = (int64_t)key_bits(keys[mid], L.off_band, L.off_j - L.off_band);
      if (band > lim) b = mid;
      else a = mid + 1;
    }
    x12[2 * q + w] = a - lo;
  }
}

void launch_self_bounds(const U128 *keys, SeedKeyLayout L, const int64_t *lohi, int npair, int64_t cd_lo,
                        int64_t cd_hi, int64_t *x12, cudaStream_t st) {
  if (npair <= 0) return;
  k_self_bounds<<<(npair + 127) / 128, 128, 0, st>>>(keys, L, lohi, npair, cd_lo, cd_hi, x12);
}

void launch_numeric(const uint8_t *bps, const int64_t *clen, const int64_t *boff, const int64_t *soff, int ncontig,
                    uint8_t *fwd, uint8_t *rc, cudaStream_t st) {
  if (ncontig <= 0) return;
  dim3 g(64, ncontig);
  k_numeric<<<g, 256, 0, st>>>(bps, clen, boff, soff, ncontig, fwd, rc);
}

__device__ __forceinline__ bool pair_hostbound(const int64_t *pstart, const int32_t *pab, int64_t np, int64_t nseeds,
                                               int comp, int64_t rs, int64_t p, int64_t *size) {
  const int64_t lo = pstart[p], hi = p + 1 < np ? pstart[p + 1] : nseeds;
  *size = hi - lo;
  return (comp == 0 && pab[2 * p] == pab[2 * p + 1]) || (rs > 0 && hi - lo > rs);
}

__global__ void k_pair_hostbound(const int64_t *__restrict__ pstart, const int32_t *__restrict__ pab, int64_t np,
                                 int64_t nseeds, int comp, int64_t rs, uint32_t *__restrict__ flag) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (int64_t)gridDim.x * blockDim.x) {
    int64_t size;
    flag[p] = pair_hostbound(pstart, pab, np, nseeds, comp, rs, p, &size) ? 1u : 0u;
  }
}

// out3 per host pair: seeds lo, hi and (anchor << 32 | partner)
__global__ void k_pair_gather(const int64_t *__restrict__ pstart, const int32_t *__restrict__ pab, int64_t np,
                              int64_t nseeds, const uint32_t *__restrict__ flag, const uint32_t *__restrict__ idx,
                              int64_t *__restrict__ out3) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (int64_t)gridDim.x * blockDim.x) {
    if (!flag[p]) continue;
    const int64_t q = idx[p];
    out3[3 * q] = pstart[p];
    out3[3 * q + 1] = p + 1 < np ? pstart[p + 1] : nseeds;
    out3[3 * q + 2] = ((int64_t)pab[2 * p] << 32) | (uint32_t)pab[2 * p + 1];
  }
}

// Bin of a device-planned pair: larger pairs in lower bins.
__device__ __forceinline__ uint32_t small_bin(int64_t size) {
  return (uint32_t)(SMALL_BINS - 1) - (uint32_t)(size < SMALL_BINS - 1 ? size : SMALL_BINS - 1);
}

// Whether a pair has a band block that can hold a chain passing the hit
// test (src/fastga_pipeline.c:656): the blocks are a pair's runs of
// consecutive bands taken two by two, and a band with no band just below
// or above it alone; a block can pass only if its seeds' spans (2 lcp each)
// add up to CHAIN_MIN.  So the pair is live iff some band start has, with
// the band just below it (its block with that band), or alone if there is
// none, a capped span sum of CHAIN_MIN.  The band below is found by walking
// back at most CHAIN_MIN / 2 seeds; a band that long reaches the cap on its
// own.  A pair that is not live makes no Local_Alignment call and no
// alignment, and leaves the path as it found it: it needs no task.
__global__ void k_pair_live(const uint16_t *__restrict__ info, int64_t n, const uint32_t *__restrict__ pflag,
                            const uint32_t *__restrict__ pidx, uint8_t *__restrict__ live) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint16_t v = info[i];
    if (!(v & BI_START)) continue;
    int sum = v & 0xff;
    if ((v & BI_ADJ) && sum < CHAIN_MIN) {
      int below = CHAIN_MIN;  // a band longer than the walk
      for (int64_t j = i - 1; j >= 0 && j >= i - CHAIN_MIN / 2; j--)
        if (info[j] & BI_START) {
          below = info[j] & 0xff;
          break;
        }
      sum += below;
    }
    if (sum >= CHAIN_MIN) live[pidx[i] + pflag[i] - 1] = 1;
  }
}

__global__ void k_small_hist(const int64_t *__restrict__ pstart, const int32_t *__restrict__ pab, int64_t np,
                             int64_t nseeds, int comp, int64_t rs, const uint8_t *__restrict__ live,
                             uint32_t *__restrict__ hist) {
  for (int64_t p0 = (int64_t)blockIdx.x * blockDim.x; p0 < np; p0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = p0 + threadIdx.x;
    int64_t size = 0;
    const bool small = p < np && !pair_hostbound(pstart, pab, np, nseeds, comp, rs, p, &size) && live[p];
    const uint32_t bin = small ? small_bin(size) : 0xffffffffu;
    const unsigned same = __match_any_sync(0xffffffffu, bin);
    if (small && (threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(&hist[bin], (unsigned)__popc(same));
  }
}

__global__ void k_small_scatter(const int64_t *__restrict__ pstart, const int32_t *__restrict__ pab, int64_t np,
                                int64_t nseeds, int comp, int64_t rs, const uint8_t *__restrict__ live,
                                uint32_t *__restrict__ cursor, uint64_t *__restrict__ small) {
  const int lane = threadIdx.x & 31;
  for (int64_t p0 = (int64_t)blockIdx.x * blockDim.x; p0 < np; p0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = p0 + threadIdx.x;
    int64_t size = 0;
    const bool small_p = p < np && !pair_hostbound(pstart, pab, np, nseeds, comp, rs, p, &size) && live[p];
    const uint32_t bin = small_p ? small_bin(size) : 0xffffffffu;
    const unsigned same = __match_any_sync(0xffffffffu, bin);
    const int leader = __ffs(same) - 1;
    uint32_t base = 0;
    if (small_p && lane == leader) base = atomicAdd(&cursor[bin], (unsigned)__popc(same));
    base = __shfl_sync(same, base, leader);
    if (small_p)
      small[base + __popc(same & ((1u << lane) - 1u))] = ((uint64_t)comp << 63) | (uint64_t)p;
  }
}

void launch_pair_hostbound(const int64_t *pstart, const int32_t *pab, int64_t np, int64_t nseeds, int comp, int64_t rs,
                           uint32_t *flag, cudaStream_t st) {
  if (np <= 0) return;
  k_pair_hostbound<<<(int)std::min<int64_t>((np + 255) / 256, 148 * 32), 256, 0, st>>>(pstart, pab, np, nseeds, comp,
                                                                                     rs, flag);
}

void launch_pair_gather(const int64_t *pstart, const int32_t *pab, int64_t np, int64_t nseeds, const uint32_t *flag,
                        const uint32_t *idx, int64_t *out3, cudaStream_t st) {
  if (np <= 0) return;
  k_pair_gather<<<(int)std::min<int64_t>((np + 255) / 256, 148 * 32), 256, 0, st>>>(pstart, pab, np, nseeds, flag, idx,
                                                                                  out3);
}

void launch_small_hist(const int64_t *pstart, const int32_t *pab, int64_t np, int64_t nseeds, int comp, int64_t rs,
                       const uint8_t *live, uint32_t *hist, cudaStream_t st) {
  if (np <= 0) return;
  k_small_hist<<<(int)std::min<int64_t>((np + 255) / 256, 148 * 32), 256, 0, st>>>(pstart, pab, np, nseeds, comp, rs,
                                                                                 live, hist);
}

void launch_small_scatter(const int64_t *pstart, const int32_t *pab, int64_t np, int64_t nseeds, int comp, int64_t rs,
                          const uint8_t *live, uint32_t *cursor, uint64_t *small, cudaStream_t st) {
  if (np <= 0) return;
  k_small_scatter<<<(int)std::min<int64_t>((np + 255) / 256, 148 * 32), 256, 0, st>>>(pstart, pab, np, nseeds, comp,
                                                                                     rs, live, cursor, small);
}

void launch_pair_live(const uint16_t *info, int64_t n, const uint32_t *pflag, const uint32_t *pidx, uint8_t *live,
                      cudaStream_t st) {
  if (n <= 0) return;
  k_pair_live<<<(int)std::min<int64_t>((n + 255) / 256, 148 * 32), 256, 0, st>>>(info, n, pflag, pidx, live);
}

void launch_band_info(const U128 *keys, int64_t n, SeedKeyLayout L, uint16_t *info, cudaStream_t st) {
  if (n <= 0) return;
  int g = (int)((n + 255) / 256);
  if (g > 148 * 32) g = 148 * 32;
  k_band_info<<<g, 256, 0, st>>>(keys, n, L, info);
}

void launch_pair_flags(const U128 *keys, int64_t n, SeedKeyLayout L, uint32_t *flag, cudaStream_t st) {
  if (n <= 0) return;
  int g = (int)((n + 255) / 256);
  if (g > 148 * 32) g = 148 * 32;
  k_pair_flags<<<g, 256, 0, st>>>(keys, n, L, flag);
}

void launch_pair_starts(const U128 *keys, int64_t n, SeedKeyLayout L, const uint32_t *flag, const uint32_t *idx,
                        int64_t *start, int32_t *ab, cudaStream_t st) {
  if (n <= 0) return;
  int g = (int)((n + 255) / 256);
  if (g > 148 * 32) g = 148 * 32;
  k_pair_starts<<<g, 256, 0, st>>>(keys, n, L, flag, idx, start, ab);
}


// ---- la_sort order of the surviving alignments ------------------------------
// (src/fastga_pipeline.c:1500-1515: by A contig, A begin, B contig, strand;
// ties in the pair's own output order.)  The key holds those fields, then the
// record's index, most significant first: aread (16 bits), abpos (32), bread
// (16) | comp (1), rank (31), index (32).

__global__ void k_aln_keys(const AlnRec *__restrict__ r, int64_t n, U128 *__restrict__ keys) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const AlnRec &a = r[i];
    U128 k;
    k.hi = ((uint64_t)(uint16_t)a.aread << 48) | ((uint64_t)(uint32_t)a.abpos << 16) | (uint64_t)(uint16_t)a.bread;
    k.lo = ((uint64_t)(a.comp & 1) << 63) | ((uint64_t)((uint32_t)a.rank & 0x7fffffffu) << 32) | (uint64_t)(uint32_t)i;
    keys[i] = k;
  }
}

// out[i] = the record of sorted key i; len[i] its trace bytes.
__global__ void k_aln_gather(const U128 *__restrict__ keys, int64_t n, const AlnRec *__restrict__ in,
                             AlnRec *__restrict__ out, int64_t *__restrict__ len) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const AlnRec a = in[(uint32_t)keys[i].lo];
    out[i] = a;
    len[i] = a.tlen;
  }
}

// One warp per record: its trace bytes to their place in sorted order; the
// record's toff becomes that place.
__global__ void k_aln_traces(AlnRec *__restrict__ recs, const int64_t *__restrict__ off, int64_t n,
                             const uint8_t *__restrict__ src, uint8_t *__restrict__ dst) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = w0; i < n; i += nw) {
    const int64_t from = recs[i].toff, to = off[i];
    const int len = recs[i].tlen;
    for (int b = lane; b < len; b += 32) dst[to + b] = src[from + b];
    __syncwarp();
    if (lane == 0) recs[i].toff = to;
  }
}

void launch_aln_keys(const AlnRec *r, int64_t n, U128 *keys, cudaStream_t st) {
  if (n <= 0) return;
  const int g = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_aln_keys<<<g, 256, 0, st>>>(r, n, keys);
}
void launch_aln_gather(const U128 *keys, int64_t n, const AlnRec *in, AlnRec *out, int64_t *len, cudaStream_t st) {
  if (n <= 0) return;
  const int g = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_aln_gather<<<g, 256, 0, st>>>(keys, n, in, out, len);
}
void launch_aln_traces(AlnRec *recs, const int64_t *off, int64_t n, const uint8_t *src, uint8_t *dst,
                       cudaStream_t st) {
  if (n <= 0) return;
  const int g = (int)std::min<int64_t>((n + 7) / 8, 148 * 16);
  k_aln_traces<<<g, 256, 0, st>>>(recs, off, n, src, dst);
}

}  // namespace pga
