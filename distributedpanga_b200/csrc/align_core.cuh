// FastGA's chain driver for one (anchor, partner) contig pair, shared by the
// device kernels and the host test harness: constants, the candidate arena,
// the band-block chain scan and what happens when a chain ends (the hit
// test, Local_Alignment calls along the chain's antidiagonal span, the
// length / error filter).  Local_Alignment itself is a template parameter
// (the device's warp aligner in align_warp.cuh; the host harness uses the
// oracle's scalar restatement), and the pair's finishing step is in
// finish.cuh.
//
// Restates, for one pair:
//   align_contigs (band blocks, chaining, window calls, filter)
//                                                   src/fastga_pipeline.c:576-813
//   Compress_TraceTo8                               lib/align.c:3892-3910
//
// Seeds are read from decoded fields instead of swide bytes; candidates and
// their trace bytes live in caller-provided arenas of fixed capacity
// (overflow sets an error bit so the caller can rerun the pair with more
// room).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define PGA_HD __host__ __device__ __forceinline__
#else
#define PGA_HD inline
#endif

namespace pga {
namespace aln {

// lib/align.c:164-183
// Entries of the alignment launch's per-SM long-call flags (above any SM id).
constexpr unsigned SM_FLAGS = 1024;
constexpr int TRIM_LEN = 15;
constexpr int DUB_TRIM = 45;
constexpr int PATH_LEN = 60;
constexpr uint64_t PATH_TOP = 0x1000000000000000ull;
constexpr uint64_t PATH_INT = 0x0fffffffffffffffull;
constexpr int TRIM_MASK = 0x7fff;
constexpr int TRIM_MLAG = 250;
constexpr int WAVE_LAG = 70;
constexpr int I32MAX = 2147483647;

// src/fastga_pipeline.c:43-54 and the driver's externs (src/pga-mpi-merge.c:61-66)
constexpr int TSPACE = 100;
constexpr int BUCK_SHIFT = 6;
constexpr int BUCK_WIDTH = 64;
constexpr int BUCK_ANTI = 128;
constexpr int BOX_FUZZ = 10;
constexpr int CHAIN_BREAK = 2000;
constexpr int CHAIN_MIN = 170;
constexpr int ALIGN_MIN = 100;
constexpr int64_t MAX_I64 = 0x7fffffffffffffffll;

enum : int { ALN_ERR_VCAP = 1, ALN_ERR_CELLS = 2, ALN_ERR_POINTS = 4, ALN_ERR_OVLS = 8, ALN_ERR_TRACE = 16 };

// Trim tables and path parameters of New_Align_Spec (lib/align.c:222-268),
// built on the host by build_align_spec.
struct AlignSpec {
  int trace_space;
  int ave_path;
  int reach;
  const int16_t *score;  // TRIM_MASK+1 entries
  const int16_t *table;  // TRIM_MASK+1 entries
};

struct Pebble {
  int ptr, diag, diff, mark;
};

struct Path {
  int tlen, diffs, abpos, bbpos, aepos, bepos;
  int trace_off;  // start of the trace (uint16 pairs) in the aligner's trace-point arena
};

// A sequence with sentinel value 4 at [-1] and [len], NUMERIC bases 0..3.
// The device aligner also reads it 2-bit packed, 32 bases per word with the
// first base in the top bits: pf forwards, pr reversed (pr's base i is
// s[len-1-i]); both end with a zero pad word.  The host code leaves them null.
struct Seq {
  const uint8_t *s;
  int len;
  const uint64_t *pf = nullptr;
  const uint64_t *pr = nullptr;
};

// ---------------------------------------------------------------------------
// Candidate and surviving alignments of one pair.
// ---------------------------------------------------------------------------
struct Ovl {
  int abpos, aepos, bbpos, bepos, diffs, tlen;
  int64_t toff;  // trace bytes (uint8 pairs: diffs, b-delta) at OvlArena::bytes + toff
  int flags;     // ELIMINATED 0x4
};

struct OvlArena {
  Ovl *ovl;
  int *perm;
  int *tmp;  // ovl_cap ints of scratch for the finishing step's sort
  int64_t ovl_cap;
  uint8_t *bytes;
  int64_t byte_cap;
  int64_t nov;    // candidates so far
  int64_t nbyte;  // trace bytes used
  int err;
  // Device pool mode: bytes is a pool shared by all warps and [nbyte,
  // byte_cap) this warp's current chunk, refilled from *pool_next.
  unsigned long long *pool_next;
  int64_t pool_cap;

  // Room for `need` more bytes.  In pool mode `warp` says whether all 32
  // lanes call this together (else one thread does).
  PGA_HD bool reserve(int64_t need, bool warp) {
    if (nbyte + need <= byte_cap) return true;
    if (pool_next == nullptr) return false;
#if defined(__CUDA_ARCH__)
    int64_t want = need > (1 << 16) ? need : (1 << 16);
    unsigned long long b0 = 0;
    if (!warp || (threadIdx.x & 31) == 0) b0 = atomicAdd(pool_next, (unsigned long long)want);
    if (warp) b0 = __shfl_sync(0xffffffffu, b0, 0);
    if ((int64_t)b0 + want > pool_cap) return false;
    nbyte = (int64_t)b0;
    byte_cap = (int64_t)b0 + want;
    return true;
#else
    (void)warp;
    return false;
#endif
  }
};

constexpr int ELIMINATED = 0x4;

struct PairResult {
  int calls;       // real Local_Alignment calls (Pair_Calls)
  int exit_bepos;  // path.bepos when the pair finished (Pair_Bepos)
  int64_t nhit, nlas;
};

// What align_contigs does when a chain of a band block ends
// (src/fastga_pipeline.c:656-760): the hit test, then Local_Alignment calls
// along the chain's antidiagonal span, each result that is long and good
// enough kept as a candidate.  cdiag, isnew and alast are the block's; a
// chain is (cov, mix, dgmin, dgmax) relative to the block and its
// antidiagonal span [alow, ahgh].
template <class Aligner>
struct ChainSink {
  bool comp, self;
  const Seq &A, &B;
  Aligner &AL;
  Path &path;
  OvlArena &O;
  PairResult &R;
  int lane, nl;
  int64_t bmxpos, mlen, doffset, aoffset;
  int64_t cdiag;
  int isnew;
  int64_t alast;

  PGA_HD int chain(int64_t cov, int mix, int dgmin, int dgmax, int64_t alow, int64_t ahgh) {
    const int alnMin = ALIGN_MIN - 50;
    const double alnRate = 0.3 + .05;  // ALIGN_RATE + .05
    if (!(cov >= CHAIN_MIN && (mix != 1 || isnew))) return 0;
    R.nhit += 1;
    dgmin += (int)(cdiag << BUCK_SHIFT);
    dgmax += (int)(cdiag << BUCK_SHIFT);
    if (comp) {
      dgmin += (int)doffset;
      dgmax += (int)doffset;
      alow += aoffset;
      ahgh += aoffset;
    } else {
      dgmin -= (int)bmxpos;
      dgmax -= (int)bmxpos;
    }
    if (ahgh <= alast) return 0;
    if (alow < alast) alow = alast;
    ahgh -= BUCK_ANTI;
    int64_t amid;
    do {
      amid = alow + BUCK_ANTI;
      if (amid > ahgh) {
        amid = ahgh;
        if (amid + dgmin < 0) {
          dgmin = (int)-amid;
          if (dgmin > dgmax) break;
        }
      }
      int called = 0;
      if (self) {
        if (dgmin > 0) {
          if (AL.call(A, B, comp, path, dgmin, dgmax, (int)amid, dgmin - 1, -1)) return 1;
          called = 1;
        } else if (dgmax < 0) {
          if (AL.call(A, B, comp, path, dgmin, dgmax, (int)amid, -1, -(dgmax + 1))) return 1;
          called = 1;
        } else
          path.abpos = path.aepos = 0;
      } else {
        if (AL.call(A, B, comp, path, dgmin, dgmax, (int)amid, -1, -1)) return 1;
        called = 1;
      }
      R.calls += called;
      int rlen = path.aepos - path.abpos;
      if (rlen >= alnMin && alnRate * rlen >= path.diffs) {
        if (O.nov >= O.ovl_cap) {
          O.err |= ALN_ERR_OVLS;
          return 1;
        }
        if (!O.reserve(path.tlen, nl > 1)) {
          O.err |= ALN_ERR_TRACE;
          return 1;
        }
        if (lane == 0) {
          Ovl &c = O.ovl[O.nov];
          c.abpos = path.abpos;
          c.aepos = path.aepos;
          c.bbpos = path.bbpos;
          c.bepos = path.bepos;
          c.diffs = path.diffs;
          c.tlen = path.tlen;
          c.flags = 0;
          c.toff = O.nbyte;
        }
        O.nov++;
        const uint16_t *tr = AL.points() + path.trace_off;  // Compress_TraceTo8
        for (int q = lane; q < path.tlen; q += nl) O.bytes[O.nbyte + q] = (uint8_t)tr[q];
        O.nbyte += path.tlen;
        R.nlas += 1;
      }
      int64_t eant = comp ? mlen - (path.abpos + path.bbpos) : (int64_t)path.aepos + path.bepos;
      if (eant <= alow) alow = amid;
      else alow = eant;
    } while (alow < ahgh);
    alast = alow;
    return 0;
  }
};

// One band block (src/fastga_pipeline.c:620-770), one seed at a time: the
// seeds of band cdiag ([b, m), stream 1) and cdiag+1 ([m, e), stream 2)
// merged by antidiagonal (stream 1 first on ties), cut into chains where a
// seed starts CHAIN_BREAK or more past the highest chain end so far.  A
// chain's coverage is the union length of its [anti, anti + 2 lcp) spans,
// mix the streams it draws on, dgmin / dgmax the extremes of its seeds'
// low diagonal bits (+BUCK_WIDTH in stream 2).
template <class Cursor, class Sink>
PGA_HD int scan_block_scalar(Cursor &C1, Cursor &C2, int64_t b, int64_t m, int64_t e, Sink &K) {
  int mix = 0, dgmin = 2 * BUCK_WIDTH, dgmax = 0;
  int64_t cov = 0, ahgh = -CHAIN_BREAK, alow = 0;
  int64_t s = b, t = m;
  int64_t ipost = C1.anti(s);
  int64_t apost = t < e ? C2.anti(t) : MAX_I64;
  while (s < m || t < e) {
    int lcp, dg, wch;
    int64_t anti;
    if (apost < ipost) {
      lcp = C2.lcp(t);
      dg = C2.dlow(t) + BUCK_WIDTH;
      anti = apost;
      t += 1;
      apost = (t >= e) ? MAX_I64 : C2.anti(t);
      wch = 0x2;
    } else {
      lcp = C1.lcp(s);
      dg = C1.dlow(s);
      anti = ipost;
      s += 1;
      ipost = (s >= m) ? MAX_I64 : C1.anti(s);
      wch = 0x1;
    }
    lcp <<= 1;
    if (anti < ahgh + CHAIN_BREAK) {
      int64_t cps = anti + lcp;
      if (cps > ahgh) {
        if (anti >= ahgh) cov += lcp;
        else cov += cps - ahgh;
        ahgh = cps;
      }
      mix |= wch;
      if (dg < dgmin) dgmin = dg;
      else if (dg > dgmax) dgmax = dg;
    } else {
      if (K.chain(cov, mix, dgmin, dgmax, alow, ahgh)) return 1;
      cov = lcp;
      ahgh = anti + lcp;
      mix = wch;
      alow = anti;
      dgmin = dgmax = dg;
    }
  }
  return K.chain(cov, mix, dgmin, dgmax, alow, ahgh);
}

// Seeds of one (anchor, partner) pair in diagonal-sort order, decoded into
// arrays (host harness).  Any type with the same interface works: band(i),
// band_end(i, band) = the first index >= i whose band differs (or n), and
// scan_block(b, m, e, sink), which runs a block's chains into the sink.
struct PairSeeds {
  const int64_t *anti_;
  const int64_t *band_;
  const uint8_t *lcp_;
  const uint8_t *dlow_;
  int64_t n;
  PGA_HD int64_t anti(int64_t i) const { return anti_[i]; }
  PGA_HD int64_t band(int64_t i) const { return band_[i]; }
  PGA_HD int lcp(int64_t i) const { return lcp_[i]; }
  PGA_HD int dlow(int64_t i) const { return dlow_[i]; }
  PGA_HD int64_t band_end(int64_t i, int64_t b) const {
    while (i < n && band_[i] == b) i++;
    return i;
  }
  struct Cursor {
    const PairSeeds *S;
    PGA_HD int64_t anti(int64_t i) { return S->anti_[i]; }
    PGA_HD int lcp(int64_t i) { return S->lcp_[i]; }
    PGA_HD int dlow(int64_t i) { return S->dlow_[i]; }
  };
  template <class Sink>
  PGA_HD int scan_block(int64_t b, int64_t m, int64_t e, Sink &K) const {
    Cursor C1{this}, C2{this};
    return scan_block_scalar(C1, C2, b, m, e, K);
  }
};

// align_contigs (src/fastga_pipeline.c:576-813) for one pair, leaving the
// candidates in O (the finishing step, finish.cuh, does the rest).  A is the anchor contig,
// already complemented when comp; `path` persists across pairs like the
// reference's Contig_Bundle path: a self pair whose window straddles the
// diagonal reads the bepos it holds on entry.  `lane`/`nl`: a warp runs this
// with every lane on the same values; lane 0 writes the candidate records and
// the lanes share the trace copies.
//
// [blo, bhi) limits the run to the band blocks whose first stream starts
// there (blo and bhi must be band starts: 0, n, or an index whose band
// differs from its predecessor's).  A block reads only its own two bands and
// resets its chain state, so for a pair of two different contigs -- where
// `path` carries nothing from one call to the next -- the blocks of
// consecutive ranges can run on different warps and their candidates,
// concatenated in range order, are exactly the whole run's.
template <class SeedsT, class Aligner>
PGA_HD int align_pair(const SeedsT &S, bool comp, bool self, const Seq &A, const Seq &B, int64_t amxpos,
                      int64_t maxdag, Aligner &AL, Path &path, OvlArena &O, PairResult &R, int lane = 0,
                      int nl = 1, int64_t blo = 0, int64_t bhi = -1) {
  const int64_t n = S.n;
  const int64_t alen = A.len, blen = B.len;
  R.calls = 0;
  R.nhit = 0;
  R.nlas = 0;
  R.exit_bepos = path.bepos;
  O.nov = 0;
  if (O.pool_next == nullptr) O.nbyte = 0;
  if (bhi < 0 || bhi > n) bhi = n;
  if (blo < 0) blo = 0;
  if (blo >= bhi) return 0;

  ChainSink<Aligner> K{comp, self, A, B, AL, path, O, R, lane, nl,
                       amxpos, alen + blen, alen - maxdag, alen - amxpos, 0, 0, -1};
  int64_t b = blo, e = blo, m;
  int64_t cdiag = S.band(blo);
  e = S.band_end(e, cdiag);
  // a block is "new" unless the band just below it has seeds
  int isnew = (blo == 0 || S.band(blo - 1) != cdiag - 1) ? 1 : 0;
  while (1) {
    // the block of band cdiag ([b, m)) and cdiag+1 ([m, e))
    m = e;
    e = S.band_end(e, cdiag + 1);
    int aux = e > m ? 1 : 0;
    if (isnew || aux) {
      K.cdiag = cdiag;
      K.isnew = isnew;
      K.alast = -1;
      if (S.scan_block(b, m, e, K)) return 1;
    }
    if (e >= n) break;
    if (aux) {
      b = m;
      cdiag += 1;
      isnew = 0;
    } else {
      b = e;
      cdiag = S.band(e);
      e = S.band_end(e, cdiag);
      isnew = 1;
    }
    if (b >= bhi) break;
  }
  R.exit_bepos = path.bepos;
  return 0;
}

}  // namespace aln
}  // namespace pga
