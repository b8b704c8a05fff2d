// The finishing step of one contig pair: its candidate alignments ordered by
// A start, then duplicates and contained copies removed, crossing alignments
// joined, and alignments inside another's box dropped.  This is what
// align_contigs does once a pair's chains are done
// (src/fastga_pipeline.c:815-980, with entwine at 505-570); the rules are
// stated here and computed with a warp's 32 lanes.
//
// The rules, for candidates c_0..c_{n-1} sorted stably by abpos:
//
// 1. Duplicates.  For j = n-1 down to 0, o = c_j looks at c_{j+1}, c_{j+2},
//    ... up to the first w with w.abpos >= o.aepos, skipping removed ones:
//      - same start (abpos, bbpos) and same end (aepos, bepos): w goes if
//        o.diffs < w.aepos, else o goes;
//      - same start, other end: the one that ends first in A goes (o on a tie);
//      - other start, same end: the one that starts later in A goes (o on a
//        tie);
//    and o's scan ends when o goes.
// 2. Crossings.  For j = n-1 down to 0, a surviving o = c_j looks at the
//    same window (o's end as it grows), skipping removed w and w that do not
//    overlap o in B.  The two are compared at their common trace points (see
//    `crossing`): if their B positions meet at an interior trace point, w is
//    joined onto o there (o keeps its trace up to the last meeting point, w's
//    after it, o takes w's end, w goes); otherwise, if they stay on one side
//    of each other, the shorter one goes when it lies inside the longer one's
//    box (BOX_FUZZ slack; for o inside w also o.abpos >= w.abpos - BOX_FUZZ).
//    o's scan goes on after o is removed here (it can still remove or join
//    later candidates).
//
// Survivors are the candidates never removed, in the sorted order.
#pragma once
#include "align_core.cuh"

namespace pga {
namespace aln {

// A value per lane.  On the device each lane holds its own; in host code
// (the test harness) one thread holds all 32.
template <class T>
struct LaneVal {
#if defined(__CUDA_ARCH__)
  T v;
  __device__ T at(int) const { return v; }
#else
  T v[32];
  T at(int l) const { return v[l]; }
#endif
};

// The lane operations the finishing step is written in.  On the device the
// 32 lanes of a converged warp make every call together, each for its own
// lane; in host code one thread runs lanes 0..31 in turn.  A lane function
// passed to `each` may write only locations no other lane writes in that
// call; `each` ends with the warp's memory in order.
struct Lanes {
  static constexpr int N = 32;
#if defined(__CUDA_ARCH__)
  __device__ static int me() { return threadIdx.x & 31; }
  template <class F>
  __device__ auto make(F f) const -> LaneVal<decltype(f(0))> {
    return LaneVal<decltype(f(0))>{f(me())};
  }
  __device__ unsigned ballot(const LaneVal<bool> &x) const { return __ballot_sync(0xffffffffu, x.v); }
  __device__ int64_t sum(const LaneVal<int64_t> &x) const {
    int64_t v = x.v;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
  }
  __device__ int64_t minimum(const LaneVal<int64_t> &x) const {
    int64_t v = x.v;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      int64_t y = __shfl_xor_sync(0xffffffffu, v, o);
      v = y < v ? y : v;
    }
    return v;
  }
  // inclusive prefix sums over lanes 0..31
  __device__ LaneVal<int64_t> scan(const LaneVal<int64_t> &x) const {
    const int l = me();
    int64_t v = x.v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int64_t y = __shfl_up_sync(0xffffffffu, v, o);
      if (l >= o) v += y;
    }
    return LaneVal<int64_t>{v};
  }
  template <class F>
  __device__ void each(F f) const {
    f(me());
    __syncwarp();
  }
#else
  template <class F>
  auto make(F f) const -> LaneVal<decltype(f(0))> {
    LaneVal<decltype(f(0))> r;
    for (int l = 0; l < N; l++) r.v[l] = f(l);
    return r;
  }
  unsigned ballot(const LaneVal<bool> &x) const {
    unsigned m = 0;
    for (int l = 0; l < N; l++)
      if (x.v[l]) m |= 1u << l;
    return m;
  }
  int64_t sum(const LaneVal<int64_t> &x) const {
    int64_t v = 0;
    for (int l = 0; l < N; l++) v += x.v[l];
    return v;
  }
  int64_t minimum(const LaneVal<int64_t> &x) const {
    int64_t v = x.v[0];
    for (int l = 1; l < N; l++) v = x.v[l] < v ? x.v[l] : v;
    return v;
  }
  LaneVal<int64_t> scan(const LaneVal<int64_t> &x) const {
    LaneVal<int64_t> r;
    int64_t v = 0;
    for (int l = 0; l < N; l++) r.v[l] = (v += x.v[l]);
    return r;
  }
  template <class F>
  void each(F f) const {
    for (int l = 0; l < N; l++) f(l);
  }
#endif
};

PGA_HD int lowest_lane(unsigned m) {
#if defined(__CUDA_ARCH__)
  return __ffs(m) - 1;
#else
  return __builtin_ffs(m) - 1;
#endif
}

PGA_HD int highest_lane(unsigned m) {
#if defined(__CUDA_ARCH__)
  return 31 - __clz(m);
#else
  return 31 - __builtin_clz(m);
#endif
}

// ---------------------------------------------------------------------------
// Stable order by abpos: bottom-up merging of runs, each element's place
// found by binary search in the other run (left-run elements count the
// right run's smaller keys, right-run elements the left run's keys not
// larger, which keeps equal keys in input order).  perm gets the order;
// tmp is scratch of the same size.
// ---------------------------------------------------------------------------
template <class W>
PGA_HD void order_by_abpos(const W &L, const Ovl *ov, int *perm, int *tmp, int64_t n) {
  L.each([&](int l) {
    for (int64_t i = l; i < n; i += W::N) perm[i] = (int)i;
  });
  int *src = perm, *dst = tmp;
  for (int64_t run = 1; run < n; run <<= 1) {
    L.each([&](int l) {
      for (int64_t i = l; i < n; i += W::N) {
        const int64_t lo = (i / (2 * run)) * (2 * run);
        const int64_t mid = lo + run < n ? lo + run : n;
        const int64_t hi = lo + 2 * run < n ? lo + 2 * run : n;
        const int key = ov[src[i]].abpos;
        int64_t a, b, place;
        if (i < mid) {  // left run: the right run's keys below key
          a = mid;
          b = hi;
          while (a < b) {
            const int64_t c = (a + b) >> 1;
            if (ov[src[c]].abpos < key) a = c + 1;
            else b = c;
          }
          place = i + (a - mid);
        } else {  // right run: the left run's keys not above key
          a = lo;
          b = mid;
          while (a < b) {
            const int64_t c = (a + b) >> 1;
            if (ov[src[c]].abpos <= key) a = c + 1;
            else b = c;
          }
          place = lo + (i - mid) + (a - lo);
        }
        dst[place] = src[i];
      }
    });
    int *x = src;
    src = dst;
    dst = x;
  }
  if (src != perm)
    L.each([&](int l) {
      for (int64_t i = l; i < n; i += W::N) perm[i] = src[i];
    });
}

// Rule 1's verdict on candidate w for o: 0 keep both, 1 remove w, 2 remove
// o, 3 w starts at or past o's end in A (o's window is over).
PGA_HD int duplicate_verdict(const Ovl &o, const Ovl &w) {
  if (w.abpos >= o.aepos) return 3;
  if (w.flags & ELIMINATED) return 0;
  const bool same_start = o.abpos == w.abpos && o.bbpos == w.bbpos;
  const bool same_end = o.aepos == w.aepos && o.bepos == w.bepos;
  if (same_start && same_end) return o.diffs < w.aepos ? 1 : 2;
  if (same_start) return o.aepos > w.aepos ? 1 : 2;
  if (same_end) return o.abpos < w.abpos ? 1 : 2;
  return 0;
}

// ---------------------------------------------------------------------------
// How two overlapping alignments J and K (J.abpos <= K.abpos) lie relative
// to each other in B.  Their B positions are compared at the A positions
// where both have a value:
//   p_0      K's start, J's B position interpolated within its trace panel
//            (J's panel b-delta scaled by the A offset into the panel, over
//            the panel's A width: TSPACE, or J's first panel's width when K
//            starts in it);
//   p_1..p_m the trace-panel boundaries x_i = (K.abpos/TSPACE + i) * TSPACE
//            below min(J.aepos, K.aepos), where both B positions are exact
//            (start plus the b-deltas of the panels before);
//   p_end    the first end in A: exact for the alignment that ends there (J
//            on a tie), interpolated over TSPACE within the other's panel.
// d_t = B(K) - B(J) at each.  `side` is 0 if d_0 = 0 or some later d_t is
// 0 or of the other sign, else the d_t closest to 0 (d_0's sign kept);
// `meet` is the largest x_i of an interior point with d_i = 0, or -1.
// The interior differences are prefix sums of the per-panel b-delta
// differences, one lane per panel boundary.  Trace bytes are (diffs,
// b-delta) pairs, one per A panel starting with the alignment's first.
// ---------------------------------------------------------------------------
struct Crossing {
  int side;
  int meet;
};

template <class W>
PGA_HD Crossing crossing(const W &L, const Ovl &J, const uint8_t *jt, const Ovl &K, const uint8_t *kt) {
  const int jp0 = J.abpos / TSPACE, kp0 = K.abpos / TSPACE, shift = kp0 - jp0;
  const int aend = J.aepos < K.aepos ? J.aepos : K.aepos;
  int m = (aend - 1) / TSPACE - kp0;  // interior boundaries
  if (m < 0) m = 0;
  // J's B position at A = kp0 * TSPACE (J's start when shift = 0)
  const int jb = J.bbpos + (int)L.sum(L.make([&](int l) -> int64_t {
    int64_t s = 0;
    for (int q = l; q < shift; q += W::N) s += jt[2 * q + 1];
    return s;
  }));
  int y0;
  if (shift == 0)
    y0 = jb + (jt[1] * (K.abpos - J.abpos)) / ((kp0 + 1) * TSPACE - J.abpos);
  else
    y0 = jb + (jt[2 * shift + 1] * (K.abpos - kp0 * TSPACE)) / TSPACE;
  const int64_t d0 = K.bbpos - y0;
  const int sgn = d0 > 0 ? 1 : (d0 < 0 ? -1 : 0);
  bool flat = sgn == 0;  // some d_t was 0 or of the other sign
  int64_t closest = d0 < 0 ? -d0 : d0;
  int meet = -1;
  // d_i = (K.bbpos - jb) + sum_{r < i} (K's b-delta r - J's b-delta shift + r)
  int64_t dm = K.bbpos - jb;  // d at the last boundary done
  int64_t ksum = 0;           // K's b-deltas of the panels done
  for (int c = 0; c < m; c += W::N) {
    const LaneVal<int64_t> step = L.make([&](int l) -> int64_t {
      const int r = c + l;
      return r < m ? (int64_t)kt[2 * r + 1] - (int64_t)jt[2 * (shift + r) + 1] : 0;
    });
    const LaneVal<int64_t> pre = L.scan(step);
    const int64_t at = dm;
    const unsigned zero = L.ballot(L.make([&](int l) { return c + l < m && at + pre.at(l) == 0; }));
    const unsigned other = L.ballot(L.make([&](int l) {
      const int64_t d = at + pre.at(l);
      return c + l < m && (sgn > 0 ? d <= 0 : d >= 0);
    }));
    const int64_t near = L.minimum(L.make([&](int l) -> int64_t {
      const int64_t d = at + pre.at(l);
      return c + l < m ? (d < 0 ? -d : d) : ((int64_t)1 << 62);
    }));
    ksum += L.sum(L.make([&](int l) -> int64_t { return c + l < m ? (int64_t)kt[2 * (c + l) + 1] : 0; }));
    dm += L.sum(step);
    if (zero) meet = (kp0 + c + highest_lane(zero) + 1) * TSPACE;
    if (other) flat = true;
    if (near < closest) closest = near;
  }
  // the first end in A
  const int ac = (kp0 + m) * TSPACE;
  const int64_t kb = K.bbpos + ksum;  // K's B position at ac
  const int64_t jy = kb - dm;         // J's
  int64_t dend;
  if (aend == J.aepos)
    dend = (kb + (kt[2 * m + 1] * (aend - ac)) / TSPACE) - J.bepos;
  else
    dend = K.bepos - (jy + (jt[2 * (shift + m) + 1] * (aend - ac)) / TSPACE);
  if (sgn > 0 ? dend <= 0 : dend >= 0) flat = true;
  const int64_t dabs = dend < 0 ? -dend : dend;
  if (dabs < closest) closest = dabs;
  return Crossing{flat ? 0 : (int)(sgn * closest), meet};
}

// ---------------------------------------------------------------------------
// The finishing step of one pair's candidates O.ovl[0..O.nov): on return
// O.perm[0..nov) is the stable abpos order and the survivors are the
// candidates without ELIMINATED; joined candidates point at new trace bytes
// taken from O's arena.  Every lane calls it with the same O (on the host,
// one thread).  On an arena overflow O.err gets ALN_ERR_TRACE.
// ---------------------------------------------------------------------------
template <class W>
PGA_HD void finish_candidates(const W &L, OvlArena &O) {
  const int64_t n = O.nov;
  Ovl *ov = O.ovl;
  int *perm = O.perm;
  order_by_abpos(L, ov, perm, O.tmp, n);

  // rule 1, 32 candidates at a time: the verdicts of a window are
  // independent (o is fixed, each w seen once), so every w up to the first
  // candidate that ends o's scan is decided together
  for (int64_t j = n - 1; j >= 0; j--) {
    const int oi = perm[j];
    const Ovl o = ov[oi];
    for (int64_t k0 = j + 1; k0 < n; k0 += W::N) {
      const LaneVal<int> v = L.make([&](int l) { return k0 + l < n ? duplicate_verdict(o, ov[perm[k0 + l]]) : 3; });
      const unsigned ends = L.ballot(L.make([&](int l) { return v.at(l) >= 2; }));
      const int lim = ends ? lowest_lane(ends) : W::N;
      L.each([&](int l) {
        if (l < lim && v.at(l) == 1) ov[perm[k0 + l]].flags |= ELIMINATED;
      });
      if (ends) {
        if (k0 + lim < n && duplicate_verdict(o, ov[perm[k0 + lim]]) == 2)
          L.each([&](int l) {
            if (l == 0) ov[oi].flags |= ELIMINATED;
          });
        break;
      }
    }
  }

  // rule 2: the next candidate that needs the crossing test is found 32 at
  // a time; the tests themselves run in order, o changing when it joins one
  for (int64_t j = n - 1; j >= 0; j--) {
    const int oi = perm[j];
    if (ov[oi].flags & ELIMINATED) continue;
    int64_t k = j + 1;
    while (k < n) {
      const Ovl o = ov[oi];
      const unsigned past = L.ballot(L.make([&](int l) { return k + l >= n || ov[perm[k + l]].abpos >= o.aepos; }));
      const int lim = past ? lowest_lane(past) : W::N;
      unsigned need = L.ballot(L.make([&](int l) {
        if (l >= lim) return false;
        const Ovl &w = ov[perm[k + l]];
        return !(w.flags & ELIMINATED) && o.bepos > w.bbpos && o.bbpos < w.bepos;
      }));
      if (!need) {
        if (past) break;
        k += W::N;
        continue;
      }
      const int64_t kk = k + lowest_lane(need);
      const int wi = perm[kk];
      const Ovl w = ov[wi];
      const uint8_t *otr = O.bytes + o.toff, *wtr = O.bytes + w.toff;
      const Crossing x = crossing(L, o, otr, w, wtr);
      if (x.meet != -1) {
        // join w onto o at the last meeting point
        const int ocut = 2 * ((x.meet - o.abpos - 1) / TSPACE + 1);
        const int wcut = 2 * ((x.meet - w.abpos - 1) / TSPACE + 1);
        const int ntlen = ocut + (w.tlen - wcut);
        if (!O.reserve(ntlen, W::N > 1)) {
          O.err |= ALN_ERR_TRACE;
          return;
        }
        uint8_t *nt = O.bytes + O.nbyte;
        L.each([&](int l) {
          for (int q = l; q < ntlen; q += W::N) nt[q] = q < ocut ? otr[q] : wtr[wcut + q - ocut];
        });
        const int64_t diffs = L.sum(L.make([&](int l) -> int64_t {
          int64_t s = 0;
          for (int q = 2 * l; q < ntlen; q += 2 * W::N) s += nt[q];
          return s;
        }));
        const int64_t toff = O.nbyte;
        O.nbyte += ntlen;
        L.each([&](int l) {
          if (l == 0) {
            Ovl &u = ov[oi];
            u.toff = toff;
            u.tlen = ntlen;
            u.diffs = (int)diffs;
            u.aepos = w.aepos;
            u.bepos = w.bepos;
            ov[wi].flags |= ELIMINATED;
          }
        });
      } else if (x.side != 0) {
        const int olen = o.aepos - o.abpos, wlen = w.aepos - w.abpos;
        int gone = -1;
        if (olen + BOX_FUZZ >= wlen) {
          if (w.aepos <= o.aepos + BOX_FUZZ && w.bbpos >= o.bbpos - BOX_FUZZ && w.bepos <= o.bepos + BOX_FUZZ)
            gone = wi;
        } else if (o.aepos <= w.aepos + BOX_FUZZ && o.bbpos >= w.bbpos - BOX_FUZZ &&
                   o.bepos <= w.bepos + BOX_FUZZ && o.abpos >= w.abpos - BOX_FUZZ) {
          gone = oi;
        }
        if (gone >= 0)
          L.each([&](int l) {
            if (l == 0) ov[gone].flags |= ELIMINATED;
          });
      }
      k = kk + 1;
    }
  }
}

}  // namespace aln
}  // namespace pga
