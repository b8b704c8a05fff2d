// Warp-cooperative wave extension: forward_wave / reverse_wave /
// Local_Alignment (lib/align.c:352-1576) with the 32 lanes of a warp
// updating the diagonals of a wave in parallel.
//
// The sequential loop of the reference visits the diagonals of a wave in one
// order (forward: k = hgh..low, reverse: k = low..hgh) and reads, for k, the
// previous wave's values at k-1, k and k+1.  Every lane here reads those from
// the previous wave's buffer (the ring buffers are double-buffered), so the
// new values equal the reference's.  What the reference accumulates in visit
// order is rebuilt with warp scans in visit order (lane 0 = first visited):
//   besta / bestx       running maximum (minimum in reverse): a diagonal is a
//                       record if it beats the maximum before it
//   lasta / trim*       the last record that passes the path-average and trim
//                       table tests
//   aclip / bclip       the last / extreme diagonal that met a sentinel
//   pebbles             every lane counts its new trace pebbles, a warp scan
//                       gives their slots in a global pool (slot numbers only
//                       name pebbles; the linked chains are the reference's)
// The rest of a wave step (boundaries, clipping, WAVE_LAG pruning) and the
// final trace-back are the reference's sequential code, run by all lanes on
// lane-uniform values.
#pragma once
#include <stdint.h>
#include "align_core.cuh"

namespace pga {
namespace aln {

constexpr uint32_t FULL = 0xffffffffu;

// Pebble pool shared by all warps of a launch: bump allocation in chunks.
struct PebblePool {
  Pebble *cells;
  unsigned long long *next;  // next free pebble (global counter)
  int64_t cap;
};

struct WarpWork {
  int *V[2], *M[2], *HA[2], *HM[2];  // HM: mark of pebble HA (marks never change once written)
  uint64_t *T[2];
  int *NA;
  int vcap;
  uint16_t *points;
  int64_t point_cap;
  PebblePool pool;
  int64_t chunk_next, chunk_end;  // this warp's current pebble chunk (lane-uniform)
  int err;
  int64_t waves, cells;  // waves after the 0-wave, and their diagonals (lane-uniform counts)
  unsigned *smflag;      // per SM id: a warp there runs a long call (null: not kept)
  int long_waves;        // waves of one wave loop that make a call long (0: never)
  int flagged;           // this warp has flagged its SM
  long long la_cycles;   // SM cycles spent in Local_Alignment calls (lane-uniform)
};

constexpr int PEBBLE_CHUNK = 4096;

// Reserve `cnt` consecutive pebbles for the warp (lane-uniform call).
__device__ __forceinline__ int64_t warp_pebbles(WarpWork &W, int cnt) {
  if (cnt == 0) return 0;
  if (W.chunk_next + cnt > W.chunk_end) {
    int64_t want = cnt > PEBBLE_CHUNK ? cnt : PEBBLE_CHUNK;
    unsigned long long base = 0;
    if ((threadIdx.x & 31) == 0) base = atomicAdd(W.pool.next, (unsigned long long)want);
    base = __shfl_sync(FULL, base, 0);
    if ((int64_t)base + want > W.pool.cap) {
      W.err |= ALN_ERR_CELLS;
      return -1;
    }
    W.chunk_next = (int64_t)base;
    W.chunk_end = (int64_t)base + want;
  }
  int64_t s = W.chunk_next;
  W.chunk_next += cnt;
  return s;
}

__device__ __forceinline__ int warp_excl_sum(int v, int lane) {
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  return x - v;
}

__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

// exclusive running max (forward) in lane order, seeded with `init`
__device__ __forceinline__ int warp_excl_max(int v, int lane, int init) {
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x = max(x, y);
  }
  int ex = __shfl_up_sync(FULL, x, 1);
  if (lane == 0) ex = init;
  return max(ex, init);
}

__device__ __forceinline__ int warp_excl_min(int v, int lane, int init) {
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x = min(x, y);
  }
  int ex = __shfl_up_sync(FULL, x, 1);
  if (lane == 0) ex = init;
  return min(ex, init);
}

__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(FULL, v, o));
  return v;
}
__device__ __forceinline__ int warp_min(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(FULL, v, o));
  return v;
}

// Highest lane with a set bit (the last in visit order), -1 if none.
__device__ __forceinline__ int last_lane(uint32_t ballot) { return ballot ? 31 - __clz(ballot) : -1; }

// 32 bases of a packed sequence starting at base o.
__device__ __forceinline__ uint64_t bases32(const uint64_t *p, int o) {
  int w = o >> 5, sh = (o & 31) << 1;
  uint64_t v = p[w];
  return sh ? (v << sh) | (p[w + 1] >> (64 - sh)) : v;
}

// Matching run of two packed sequences from offsets oa, ob, at most mx bases.
__device__ __forceinline__ int match_run(const uint64_t *pa, int oa, const uint64_t *pb, int ob, int mx) {
  int t = 0;
  while (t < mx) {
    uint64_t d = bases32(pa, oa + t) ^ bases32(pb, ob + t);
    int chunk = mx - t < 32 ? mx - t : 32;
    if (d) {
      int lead = __clzll(d) >> 1;
      if (lead < chunk) return t + lead;
    }
    t += chunk;
  }
  return mx;
}

// Forward snake along diagonal k from a-position x (A[x..], B[x-k..]): the
// reference's byte loop stops at the first mismatch, or at B's sentinel
// (B[blen], checked first) or A's (A[alen]).  Starts outside the sequences
// count as meeting that sequence's sentinel, so no read leaves the buffers.
__device__ __forceinline__ int snake_fwd(const Seq &A, const Seq &B, int x, int k, int *hitb, int *hita) {
  int y = x - k;
  *hitb = *hita = 0;
  if (y < 0 || y > B.len) {
    *hitb = 1;
    return x;
  }
  if (x < 0 || x > A.len) {
    *hita = 1;
    return x;
  }
  int ra = A.len - x, rb = B.len - y;
  int mx = ra < rb ? ra : rb;
  int t = match_run(A.pf, x, B.pf, y, mx);
  if (t == mx) {
    if (rb <= ra) *hitb = 1;
    else *hita = 1;
  }
  return x + t;
}

// Reverse snake along diagonal k from x: compares A[x-1], A[x-2], .. with
// B[x-k-1], ..; sentinels A[-1] and B[-1] (read through the reversed copies).
__device__ __forceinline__ int snake_rev(const Seq &A, const Seq &B, int x, int k, int *hitb, int *hita) {
  int y = x - k;
  *hitb = *hita = 0;
  if (y <= 0 || y >= B.len + 1) {  // B[-1], B[blen] or outside
    *hitb = 1;
    return x;
  }
  if (x <= 0 || x > A.len) {
    *hita = 1;
    return x;
  }
  int ra = x, rb = y;
  int mx = ra < rb ? ra : rb;
  int t = match_run(A.pr, A.len - x, B.pr, B.len - y, mx);
  if (t == mx) {
    if (rb <= ra) *hitb = 1;
    else *hita = 1;
  }
  return x - t;
}

// The reference shifts one 1 into the match history b per matched base and
// counts m up while b's PATH_TOP bit is clear (lib/align.c:663-668): the
// closed form for a run of r bases.
__device__ __forceinline__ void history_run(uint64_t &b, int &m, int r) {
  if (r <= 0) return;
  int L = r < 61 ? r : 61;
  uint64_t mask = ((1ull << L) - 1) << (61 - L);
  m += L - __popcll(b & mask);
  b = r >= 64 ? ~0ull : ((b << r) | ((1ull << r) - 1));
}

// ---------------------------------------------------------------------------
// One wave of forward_wave / reverse_wave after its boundary diagonals are
// set: every diagonal of [low, hgh] computed from the previous wave's buffer
// (cur) into the other buffer, in the reference's visit order (forward:
// k = hgh..low, reverse: k = low..hgh).
//
// Each lane takes up to WJ consecutive diagonals of the visit order (lane 0
// the first), so a wave of up to 32*WJ diagonals is one pass: the lane's
// loads and snakes are independent and run side by side, and the visit-order
// scans are a lane-local pass plus one warp scan.  Wider waves take several
// passes, carried in visit order.
// ---------------------------------------------------------------------------
constexpr int WJ = 4;

// What a one-pass sweep leaves in registers for wave_prune.
struct WaveSlice {
  int c[WJ];
  int k0;       // the lane's first diagonal
  int nact;     // its diagonals
  bool single;  // one pass covered [low, hgh]
};

// Lockstep snakes of a lane's diagonals: forward along A.pf / B.pf from
// (x, x-k), reverse along A.pr / B.pr from (A.len-x, B.len-y); stops and
// sentinel hits as snake_fwd / snake_rev.
template <int J>
__device__ __forceinline__ void lane_snakes(const bool FWD, const Seq &A, const Seq &B, int nact, const int *k, int *x,
                                            int *run, int *hb, int *hA) {
  int oa[J], ob[J], mx[J], t[J];
  bool go[J];
#pragma unroll
  for (int j = 0; j < J; j++) {
    go[j] = false;
    hb[j] = hA[j] = 0;
    t[j] = 0;
    mx[j] = 0;
    oa[j] = ob[j] = 0;
    if (j < nact) {
      int xx = x[j], y = xx - k[j];
      if (FWD) {
        if (y < 0 || y > B.len) hb[j] = 1;
        else if (xx < 0 || xx > A.len) hA[j] = 1;
        else {
          int ra = A.len - xx, rb = B.len - y;
          mx[j] = ra < rb ? ra : rb;
          oa[j] = xx;
          ob[j] = y;
          go[j] = mx[j] > 0;
        }
      } else {
        if (y <= 0 || y >= B.len + 1) hb[j] = 1;
        else if (xx <= 0 || xx > A.len) hA[j] = 1;
        else {
          mx[j] = xx < y ? xx : y;
          oa[j] = A.len - xx;
          ob[j] = B.len - y;
          go[j] = mx[j] > 0;
        }
      }
    }
  }
  const uint64_t *pa = FWD ? A.pf : A.pr, *pb = FWD ? B.pf : B.pr;
  bool any = false;
#pragma unroll
  for (int j = 0; j < J; j++) any |= go[j];
  while (any) {
    any = false;
#pragma unroll
    for (int j = 0; j < J; j++) {
      if (go[j]) {
        uint64_t d = bases32(pa, oa[j] + t[j]) ^ bases32(pb, ob[j] + t[j]);
        int chunk = mx[j] - t[j] < 32 ? mx[j] - t[j] : 32;
        int lead = d ? (__clzll(d) >> 1) : 32;
        if (lead < chunk) {
          t[j] += lead;
          go[j] = false;
        } else {
          t[j] += chunk;
          go[j] = t[j] < mx[j];
        }
        any |= go[j];
      }
    }
  }
#pragma unroll
  for (int j = 0; j < J; j++) {
    if (j < nact && !hb[j] && !hA[j]) {
      if (t[j] == mx[j]) {
        int xx = x[j], y = xx - k[j];
        int ra = FWD ? A.len - xx : xx, rb = FWD ? B.len - y : y;
        if (rb <= ra) hb[j] = 1;
        else hA[j] = 1;
      }
      x[j] = FWD ? x[j] + t[j] : x[j] - t[j];
    }
    run[j] = t[j];
  }
}

// 32 bases of a packed sequence from a 2-bit shift sh (0..62) into words
// (w0, w1): w0 << sh with w1's top bits shifted in, no branch on sh == 0.
__device__ __forceinline__ uint64_t join32(uint64_t w0, uint64_t w1, int sh) {
  return (w0 << sh) | ((w1 >> 1) >> (63 - sh));
}

// The snake of one diagonal (the one-diagonal-per-lane case of
// lane_snakes): the same stops and sentinel hits, 64 bases per round from
// three words of each packed sequence loaded together.  The third word may
// lie past this sequence's copy (its bases are beyond mx and never count);
// the packed buffer has spare words at its end.
__device__ __forceinline__ void snake1(const bool FWD, const Seq &A, const Seq &B, bool act, int k, int &x, int &run,
                                       int &hb, int &hA) {
  hb = hA = 0;
  run = 0;
  if (!act) return;
  const int y = x - k;
  int oa, ob, mx;
  const uint64_t *pa, *pb;
  if (FWD) {
    if (y < 0 || y > B.len) {
      hb = 1;
      return;
    }
    if (x < 0 || x > A.len) {
      hA = 1;
      return;
    }
    const int ra = A.len - x, rb = B.len - y;
    mx = ra < rb ? ra : rb;
    oa = x;
    ob = y;
    pa = A.pf;
    pb = B.pf;
  } else {
    if (y <= 0 || y >= B.len + 1) {
      hb = 1;
      return;
    }
    if (x <= 0 || x > A.len) {
      hA = 1;
      return;
    }
    mx = x < y ? x : y;
    oa = A.len - x;
    ob = B.len - y;
    pa = A.pr;
    pb = B.pr;
  }
  int t = 0;
  while (t < mx) {
    const int qa = oa + t, qb = ob + t;
    const uint64_t *ua = pa + (qa >> 5), *ub = pb + (qb >> 5);
    const int sa = (qa & 31) << 1, sb = (qb & 31) << 1;
    const uint64_t a0 = ua[0], a1 = ua[1], a2 = ua[2], b0 = ub[0], b1 = ub[1], b2 = ub[2];
    const uint64_t d0 = join32(a0, a1, sa) ^ join32(b0, b1, sb);
    const uint64_t d1 = join32(a1, a2, sa) ^ join32(b1, b2, sb);
    const int lead = d0 ? (__clzll(d0) >> 1) : 32 + (d1 ? (__clzll(d1) >> 1) : 32);
    const int chunk = mx - t < 64 ? mx - t : 64;
    if (lead < chunk) {
      t += lead;
      break;
    }
    t += chunk;
  }
  if (t == mx) {
    const int ra = FWD ? A.len - x : x, rb = FWD ? B.len - y : y;
    if (rb <= ra) hb = 1;
    else hA = 1;
  }
  x = FWD ? x + t : x - t;
  run = t;
}

// v[j] for a per-lane index j < J, without local memory
template <int J>
__device__ __forceinline__ int pick(const int *v, int j) {
  int r = v[0];
#pragma unroll
  for (int q = 1; q < J; q++)
    if (j == q) r = v[q];
  return r;
}

// One pass of a wave over visit positions [p0, p0 + 32*J): lane l takes
// positions p0 + l*J .. p0 + l*J + J-1.  carry is the running best before
// the pass.
template <int J>
__device__ __forceinline__ int wave_pass(const bool FWD, WarpWork &W, const AlignSpec &spec, const Seq &A, const Seq &B,
                                         int low, int hgh, int w, int p0, int dif, int cur, int &carry, int &besta,
                                         int &bestx, int &lasta, int &trima, int &trimx, int &trimd, int &trimha,
                                         int &more, int &aclip, int &bclip, WaveSlice &WS) {
  const int lane = threadIdx.x & 31;
  const int vmask = W.vcap - 1;
  const int tspace = spec.trace_space;
  const int PATH_AVE = spec.ave_path;
  const int16_t *SCORE = spec.score;
  const int16_t *TABLE = spec.table;
  const int *Vo = W.V[cur], *Mo = W.M[cur], *HAo = W.HA[cur], *HMo = W.HM[cur];
  const uint64_t *To = W.T[cur];
  int *Vn = W.V[cur ^ 1], *Mn = W.M[cur ^ 1], *HAn = W.HA[cur ^ 1], *HMn = W.HM[cur ^ 1];
  uint64_t *Tn = W.T[cur ^ 1];
  int *NA = W.NA;
  Pebble *cells = W.pool.cells;
  const int pl = p0 + lane * J;
  int nact = w - pl;
  if (nact > J) nact = J;
  if (nact < 0) nact = 0;
  const int k0 = FWD ? hgh - pl : low + pl;
  int k[J], c[J], x[J], m[J], ha[J], hm[J], nak[J], run[J], hb[J], hA[J], npb[J];
  uint64_t b[J];
  // previous wave around the lane's diagonals: forward nv[i] = V[k0+1-i],
  // reverse nv[i] = V[k0-1+i]
  int nv[J + 2];
#pragma unroll
  for (int i = 0; i < J + 2; i++) {
    nv[i] = 0;
    if (nact > 0 && i < nact + 2) nv[i] = Vo[(FWD ? k0 + 1 - i : k0 - 1 + i) & vmask];
  }
#pragma unroll
  for (int j = 0; j < J; j++) {
    k[j] = FWD ? k0 - j : k0 + j;
    c[j] = x[j] = m[j] = hm[j] = nak[j] = npb[j] = 0;
    ha[j] = -1;
    b[j] = 0;
    if (j < nact) {
      int src, sk;
      if (FWD) {
        int ap = nv[j], ac = nv[j + 1], am = nv[j + 2];
        if (ac < am) src = (am < ap) ? 1 : -1;
        else src = (ac < ap) ? 1 : 0;
        c[j] = src == 1 ? ap + 1 : (src == -1 ? am + 1 : ac + 2);
      } else {
        int am = nv[j], ac = nv[j + 1], ap = nv[j + 2];
        if (ac > ap) src = (ap > am) ? -1 : 1;
        else src = (ac > am) ? -1 : 0;
        c[j] = src == -1 ? am - 1 : (src == 1 ? ap - 1 : ac - 2);
      }
      sk = k[j] + src;
      bool dflt = FWD ? (src == 1 && k[j] == hgh) : (src == -1 && k[j] == low);
      if (dflt) {
        m[j] = PATH_LEN;
        b[j] = PATH_INT;
      } else {
        int si = sk & vmask;
        m[j] = Mo[si];
        b[j] = To[si];
        ha[j] = HAo[si];
        hm[j] = HMo[si];
      }
      nak[j] = NA[k[j] & vmask];
      if ((b[j] & PATH_TOP) != 0) m[j] -= 1;
      b[j] <<= 1;
      x[j] = (c[j] + k[j]) >> 1;
    }
  }
  lane_snakes<J>(FWD, A, B, nact, k, x, run, hb, hA);
  int npl = 0;
#pragma unroll
  for (int j = 0; j < J; j++) {
    if (j < nact) {
      history_run(b[j], m[j], run[j]);
      c[j] = (x[j] << 1) - k[j];
      int hq = hm[j];
      if (FWD) {
        for (int q = nak[j]; x[j] >= q; q += tspace)
          if (hq < q) {
            npb[j]++;
            hq = q;
          }
      } else {
        for (int q = nak[j]; x[j] <= q; q -= tspace)
          if (hq > q) {
            npb[j]++;
            hq = q;
          }
      }
      npl += npb[j];
    }
  }
  // pebble slots in visit order
  int off, tot;
  if (__ballot_sync(FULL, npl > 1) == 0) {
    uint32_t one = __ballot_sync(FULL, npl == 1);
    off = __popc(one & ((1u << lane) - 1));
    tot = __popc(one);
  } else {
    off = warp_excl_sum(npl, lane);
    tot = warp_sum(npl);
  }
  int64_t pb0 = warp_pebbles(W, tot);
  if (pb0 < 0) return 1;
  int64_t s = pb0 + off;
#pragma unroll
  for (int j = 0; j < J; j++) {
    if (j < nact) {
      if (FWD) {
        while (x[j] >= nak[j]) {
          if (hm[j] < nak[j]) {
            cells[s] = {ha[j], k[j], dif, nak[j]};
            ha[j] = (int)s;
            hm[j] = nak[j];
            s += 1;
          }
          nak[j] += tspace;
        }
      } else {
        while (x[j] <= nak[j]) {
          if (hm[j] > nak[j]) {
            cells[s] = {ha[j], k[j], dif, nak[j]};
            ha[j] = (int)s;
            hm[j] = nak[j];
            s += 1;
          }
          nak[j] -= tspace;
        }
      }
      int vi = k[j] & vmask;
      NA[vi] = nak[j];
      Vn[vi] = c[j];
      Tn[vi] = b[j];
      Mn[vi] = m[j];
      HAn[vi] = ha[j];
      HMn[vi] = hm[j];
    }
  }
  // clips: bclip from the first visited diagonal that met B's end, aclip
  // from the last visited that met A's end
  int fb = -1, la = -1;
#pragma unroll
  for (int j = J - 1; j >= 0; j--)
    if (j < nact && hb[j]) fb = j;
#pragma unroll
  for (int j = 0; j < J; j++)
    if (j < nact && hA[j]) la = j;
  uint32_t bbl = __ballot_sync(FULL, fb >= 0), bal = __ballot_sync(FULL, la >= 0);
  if (bbl) {
    more = 0;
    int L = __ffs(bbl) - 1;
    int kk = __shfl_sync(FULL, FWD ? k0 - fb : k0 + fb, L);
    if (FWD ? (bclip < kk) : (bclip > kk)) bclip = kk;
  }
  if (bal) {
    more = 0;
    int L = last_lane(bal);
    aclip = __shfl_sync(FULL, FWD ? k0 - la : k0 + la, L);
  }
  // records: c beyond the running best (max forward, min reverse) in visit order
  int agg = FWD ? -2147483647 : 2147483647;
#pragma unroll
  for (int j = 0; j < J; j++)
    if (j < nact) agg = FWD ? max(agg, c[j]) : min(agg, c[j]);
  int pm = FWD ? warp_excl_max(agg, lane, carry) : warp_excl_min(agg, lane, carry);
  int lr = -1, lp = -1, lt = -1;
#pragma unroll
  for (int j = 0; j < J; j++) {
    if (j < nact) {
      bool rec = FWD ? c[j] > pm : c[j] < pm;
      if (rec) {
        pm = c[j];
        lr = j;
        if (m[j] >= PATH_AVE) {
          lp = j;
          if (TABLE[b[j] & TRIM_MASK] >= 0 && TABLE[(b[j] >> TRIM_LEN) & TRIM_MASK] + SCORE[b[j] & TRIM_MASK] >= 0)
            lt = j;
        }
      }
    }
  }
  uint32_t rb = __ballot_sync(FULL, lr >= 0);
  if (rb) {
    int L = last_lane(rb);
    carry = __shfl_sync(FULL, pick<J>(c, lr), L);
    besta = carry;
    bestx = __shfl_sync(FULL, pick<J>(x, lr), L);
    uint32_t pab = __ballot_sync(FULL, lp >= 0);
    if (pab) {
      lasta = __shfl_sync(FULL, pick<J>(c, lp), last_lane(pab));
      uint32_t trb = __ballot_sync(FULL, lt >= 0);
      if (trb) {
        int T2 = last_lane(trb);
        trima = __shfl_sync(FULL, pick<J>(c, lt), T2);
        trimx = __shfl_sync(FULL, pick<J>(x, lt), T2);
        trimd = dif;
        trimha = __shfl_sync(FULL, pick<J>(ha, lt), T2);
      }
    }
  }
  if (WS.single) {
#pragma unroll
    for (int j = 0; j < J; j++) WS.c[j] = c[j];
    WS.k0 = k0;
    WS.nact = nact;
  }
  return 0;
}

// The whole wave: one pass of single diagonals when it is at most 32 wide,
// else passes of WJ diagonals per lane.
__device__ __forceinline__ int wave_sweep(const bool FWD, WarpWork &W, const AlignSpec &spec, const Seq &A,
                                          const Seq &B, int low, int hgh, int dif, int cur, int &besta, int &bestx,
                                          int &lasta, int &trima, int &trimx, int &trimd, int &trimha, int &more,
                                          int &aclip, int &bclip, WaveSlice &WS) {
  const int w = hgh - low + 1;
  WS.single = w <= 32 * WJ;
  WS.nact = 0;
  WS.k0 = 0;
  int carry = besta;
  if (w <= 32)
    return wave_pass<1>(FWD, W, spec, A, B, low, hgh, w, 0, dif, cur, carry, besta, bestx, lasta, trima, trimx,
                             trimd, trimha, more, aclip, bclip, WS);
  for (int p0 = 0; p0 < w; p0 += 32 * WJ)
    if (wave_pass<WJ>(FWD, W, spec, A, B, low, hgh, w, p0, dif, cur, carry, besta, bestx, lasta, trima, trimx,
                           trimd, trimha, more, aclip, bclip, WS))
      return 1;
  return 0;
}

// WAVE_LAG pruning of [low, hgh] (already clipped) on the wave just made:
// hgh becomes the largest and low the smallest diagonal within WAVE_LAG of
// the best antidiagonal, or hgh = low - 1 when none is (the reference's
// loop from either end).  V is the new wave's buffer.
__device__ __forceinline__ void wave_prune(const bool FWD, const WarpWork &W, const int *V, int besta, int &low,
                                           int &hgh, const WaveSlice &WS) {
  if (hgh < low) return;
  const int vmask = W.vcap - 1;
  const int n = FWD ? besta - WAVE_LAG : besta + WAVE_LAG;
  if (WS.single) {
    int kmax = -2147483647, kmin = 2147483647;
#pragma unroll
    for (int j = 0; j < WJ; j++) {
      int k = FWD ? WS.k0 - j : WS.k0 + j;
      if (j < WS.nact && k >= low && k <= hgh && (FWD ? WS.c[j] >= n : WS.c[j] <= n)) {
        kmax = max(kmax, k);
        kmin = min(kmin, k);
      }
    }
    kmax = __reduce_max_sync(FULL, kmax);
    kmin = __reduce_min_sync(FULL, kmin);
    if (kmin <= kmax) {
      hgh = kmax;
      low = kmin;
    } else
      hgh = low - 1;
    return;
  }
  if (FWD) {
    while (hgh >= low)
      if (V[hgh & vmask] < n)
        hgh -= 1;
      else {
        while (V[low & vmask] < n) low += 1;
        break;
      }
  } else {
    while (hgh >= low)
      if (V[hgh & vmask] > n)
        hgh -= 1;
      else {
        while (V[low & vmask] > n) low += 1;
        break;
      }
  }
}

// ---------------------------------------------------------------------------
// Register-resident waves.  While a wave is at most 32 diagonals wide (and
// the previous one was not empty) diagonal k lives in lane k mod 32: its
// antidiagonal, match count, match history, head pebble, head mark and next
// trace mark stay in registers, the previous wave's neighbours come by
// shuffle, and the visit-order questions (pebble slots, records, clips,
// pruning) are answered with ballots rotated into visit order and warp
// reductions.  NA is also written through to memory; the other fields go to
// the memory ring only when a wider wave hands over to wave_sweep.
// ---------------------------------------------------------------------------
struct RegWave {
  int V, M, HA, HM, NA;
  uint64_t T;
};

// What a register wave needs of WarpWork, held in the wave loop's registers
// (WarpWork itself lives in addressable memory).
struct RegCtx {
  int vmask;
  int *NA;
  Pebble *cells;
  unsigned long long *pool_next;
  int64_t pool_cap;
  int64_t chunk_next, chunk_end;  // the warp's current pebble chunk
  int err;
};

// warp_pebbles on a RegCtx.
__device__ __forceinline__ int64_t reg_pebbles(RegCtx &X, int cnt) {
  if (cnt == 0) return 0;
  if (X.chunk_next + cnt > X.chunk_end) {
    int64_t want = cnt > PEBBLE_CHUNK ? cnt : PEBBLE_CHUNK;
    unsigned long long base = 0;
    if ((threadIdx.x & 31) == 0) base = atomicAdd(X.pool_next, (unsigned long long)want);
    base = __shfl_sync(FULL, base, 0);
    if ((int64_t)base + want > X.pool_cap) {
      X.err |= ALN_ERR_CELLS;
      return -1;
    }
    X.chunk_next = (int64_t)base;
    X.chunk_end = (int64_t)base + want;
  }
  int64_t s = X.chunk_next;
  X.chunk_next += cnt;
  return s;
}

// Visit position of lane l's diagonal (forward: hgh first, reverse: low first).
__device__ __forceinline__ int reg_pos(const bool FWD, int l, int low, int hgh) {
  return FWD ? ((hgh - l) & 31) : ((l - low) & 31);
}
__device__ __forceinline__ int reg_lane(const bool FWD, int p, int low, int hgh) {
  return FWD ? ((hgh - p) & 31) : ((low + p) & 31);
}
// A lane mask reordered so that bit p is the lane at visit position p.
__device__ __forceinline__ uint32_t reg_posmask(const bool FWD, uint32_t m, int low, int hgh) {
  return FWD ? __brev(__funnelshift_l(m, m, 31 - (hgh & 31))) : __funnelshift_r(m, m, low & 31);
}

// Memory ring (buffer cur) -> registers for the diagonals of [plow, phgh].
__device__ __forceinline__ void reg_load(const WarpWork &W, int cur, int plow, int phgh, RegWave &R) {
  const int lane = threadIdx.x & 31, vmask = W.vcap - 1;
  const int k = plow + ((lane - plow) & 31);
  if (k <= phgh) {
    const int vi = k & vmask;
    R.V = W.V[cur][vi];
    R.M = W.M[cur][vi];
    R.T = W.T[cur][vi];
    R.HA = W.HA[cur][vi];
    R.HM = W.HM[cur][vi];
    R.NA = W.NA[vi];
  }
}

// Registers -> memory ring (buffer cur) for the diagonals of [plow, phgh].
__device__ __forceinline__ void reg_store(WarpWork &W, int cur, int plow, int phgh, const RegWave &R) {
  const int lane = threadIdx.x & 31, vmask = W.vcap - 1;
  const int k = plow + ((lane - plow) & 31);
  if (k <= phgh) {
    const int vi = k & vmask;
    W.V[cur][vi] = R.V;
    W.M[cur][vi] = R.M;
    W.T[cur][vi] = R.T;
    W.HA[cur][vi] = R.HA;
    W.HM[cur][vi] = R.HM;
    W.NA[vi] = R.NA;
  }
}

// One wave in registers: [low, hgh] (at most 32 wide) from the previous
// wave [plow, phgh] (not empty, inside [low-1, hgh+1]).  Same results as
// wave_sweep; fills WS for wave_prune.
__device__ __forceinline__ int reg_wave(const bool FWD, RegCtx &X, const AlignSpec &spec, const Seq &A, const Seq &B,
                                        int low, int hgh, int plow, int phgh, int dif, RegWave &R, int &besta,
                                        int &bestx, int &lasta, int &trima, int &trimx, int &trimd, int &trimha,
                                        int &more, int &aclip, int &bclip, WaveSlice &WS) {
  const int lane = threadIdx.x & 31;
  const int vmask = X.vmask;
  const int tspace = spec.trace_space;
  const int BV = FWD ? -1 : I32MAX;
  const int k = low + ((lane - low) & 31);
  const bool act = k <= hgh;
  // the previous wave at k+1, k, k-1
  const int vp = __shfl_sync(FULL, R.V, (lane + 1) & 31), vm = __shfl_sync(FULL, R.V, (lane - 1) & 31);
  const int ap = (k + 1 >= plow && k + 1 <= phgh) ? vp : BV;
  const int ac = (k >= plow && k <= phgh) ? R.V : BV;
  const int am = (k - 1 >= plow && k - 1 <= phgh) ? vm : BV;
  int src, c;
  if (FWD) {
    if (ac < am) src = (am < ap) ? 1 : -1;
    else src = (ac < ap) ? 1 : 0;
    c = src == 1 ? ap + 1 : (src == -1 ? am + 1 : ac + 2);
  } else {
    if (ac > ap) src = (ap > am) ? -1 : 1;
    else src = (ac > am) ? -1 : 0;
    c = src == -1 ? am - 1 : (src == 1 ? ap - 1 : ac - 2);
  }
  const int sl = (k + src) & 31;
  const int sM = __shfl_sync(FULL, R.M, sl), sHA = __shfl_sync(FULL, R.HA, sl), sHM = __shfl_sync(FULL, R.HM, sl);
  const uint64_t sT = __shfl_sync(FULL, R.T, sl);
  // next trace mark: a new bottom diagonal copies the one above it, a new top
  // diagonal the one below it
  const int nlo = __shfl_sync(FULL, R.NA, plow & 31), nhi = __shfl_sync(FULL, R.NA, phgh & 31);
  const bool dflt = FWD ? (src == 1 && k == hgh) : (src == -1 && k == low);
  int m = dflt ? PATH_LEN : sM;
  uint64_t b = dflt ? PATH_INT : sT;
  int ha = dflt ? -1 : sHA, hm = dflt ? 0 : sHM;
  int nak = (k >= plow && k <= phgh) ? R.NA : (k < plow ? nlo : nhi);
  if ((b & PATH_TOP) != 0) m -= 1;
  b <<= 1;
  int x = (c + k) >> 1;
  int run[1], hb[1], hA[1];
  snake1(FWD, A, B, act, k, x, run[0], hb[0], hA[0]);
  int npb = 0;
  if (act) {
    history_run(b, m, run[0]);
    c = (x << 1) - k;
    int hq = hm;
    if (FWD) {
      for (int q = nak; x >= q; q += tspace)
        if (hq < q) {
          npb++;
          hq = q;
        }
    } else {
      for (int q = nak; x <= q; q -= tspace)
        if (hq > q) {
          npb++;
          hq = q;
        }
    }
  }
  // trim test of this diagonal's history (used if it is a record)
  bool tr = false;
  if (act && m >= spec.ave_path)
    tr = spec.table[b & TRIM_MASK] >= 0 &&
         spec.table[(b >> TRIM_LEN) & TRIM_MASK] + spec.score[b & TRIM_MASK] >= 0;
  // pebble slots in visit order
  const int pos = reg_pos(FWD, lane, low, hgh);
  int off, tot;
  if (__ballot_sync(FULL, npb > 1) == 0) {
    uint32_t one = reg_posmask(FWD, __ballot_sync(FULL, npb == 1), low, hgh);
    off = __popc(one & ((1u << pos) - 1));
    tot = __popc(one);
  } else {
    // visit-order exclusive sum over positions
    int xsum = npb;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      int y = __shfl_sync(FULL, xsum, reg_lane(FWD, pos - d, low, hgh));
      if (pos >= d) xsum += y;
    }
    off = xsum - npb;
    tot = __reduce_add_sync(FULL, npb);
  }
  int64_t pb0 = reg_pebbles(X, tot);
  if (pb0 < 0) return 1;
  if (act) {
    int64_t s = pb0 + off;
    Pebble *cells = X.cells;
    if (FWD) {
      while (x >= nak) {
        if (hm < nak) {
          cells[s] = {ha, k, dif, nak};
          ha = (int)s;
          hm = nak;
          s += 1;
        }
        nak += tspace;
      }
    } else {
      while (x <= nak) {
        if (hm > nak) {
          cells[s] = {ha, k, dif, nak};
          ha = (int)s;
          hm = nak;
          s += 1;
        }
        nak -= tspace;
      }
    }
    X.NA[k & vmask] = nak;
    R.V = c;
    R.M = m;
    R.T = b;
    R.HA = ha;
    R.HM = hm;
    R.NA = nak;
  }
  // clips: bclip from the first visited diagonal that met B's end, aclip
  // from the last visited that met A's end
  const uint32_t hbm = reg_posmask(FWD, __ballot_sync(FULL, act && hb[0]), low, hgh);
  const uint32_t ham = reg_posmask(FWD, __ballot_sync(FULL, act && hA[0]), low, hgh);
  if (hbm) {
    more = 0;
    const int p = __ffs(hbm) - 1;
    const int kb = FWD ? hgh - p : low + p;
    if (FWD ? (bclip < kb) : (bclip > kb)) bclip = kb;
  }
  if (ham) {
    more = 0;
    const int p = 31 - __clz(ham);
    aclip = FWD ? hgh - p : low + p;
  }
  // records: c beyond the running best in visit order.  The last record is
  // the first diagonal reaching the wave's best; the one before it the first
  // reaching the best of the earlier positions, and so on.
  const int carry = besta;
  const int cv = act ? c : (FWD ? -2147483647 : 2147483647);
  int best = FWD ? __reduce_max_sync(FULL, cv) : __reduce_min_sync(FULL, cv);
  if (FWD ? best > carry : best < carry) {
    const int fl = (m >= spec.ave_path ? 1 : 0) | (tr ? 2 : 0);
    int limit = 32;  // positions below this are still candidates
    int lp = -1, lt = -1;
    bool first = true;
    while (true) {
      const uint32_t eq = reg_posmask(FWD, __ballot_sync(FULL, act && c == best && pos < limit), low, hgh);
      const int p = __ffs(eq) - 1;
      const int L = reg_lane(FWD, p, low, hgh);
      if (first) {
        besta = best;
        bestx = __shfl_sync(FULL, x, L);
        first = false;
      }
      const int f = __shfl_sync(FULL, fl, L);
      if (lp < 0 && (f & 1)) lp = L;
      if (f & 2) {
        lt = L;
        break;
      }
      limit = p;
      const int cv2 = (act && pos < limit) ? c : (FWD ? -2147483647 : 2147483647);
      best = FWD ? __reduce_max_sync(FULL, cv2) : __reduce_min_sync(FULL, cv2);
      if (!(FWD ? best > carry : best < carry)) break;
    }
    if (lp >= 0) lasta = __shfl_sync(FULL, c, lp);
    if (lt >= 0) {
      trima = __shfl_sync(FULL, c, lt);
      trimx = __shfl_sync(FULL, x, lt);
      trimd = dif;
      trimha = __shfl_sync(FULL, ha, lt);
    }
  }
  WS.single = true;
  WS.c[0] = c;
  WS.k0 = k;
  WS.nact = act ? 1 : 0;
  return 0;
}

// The wave loop of forward_wave (FWD) or reverse_wave after the 0-wave:
// grow the band, compute the wave, clip at sequence ends, prune.  Waves of
// at most 32 diagonals run in registers (reg_wave), wider ones through the
// memory ring (wave_sweep).
__device__ __forceinline__ int wave_loop(const bool FWD, WarpWork &W, const AlignSpec &spec, const Seq &A, const Seq &B,
                                         const uint8_t *aseq, const uint8_t *bseq, int minp, int maxp, int &low,
                                         int &hgh, int &dif, int &cur, int &besta, int &bestx, int &lasta,
                                         int &trima, int &trimx, int &trimd, int &trimha, int &more, int &aclip,
                                         int &bclip, int &morem, int &morea, int &morex, int &mored, int &moreha,
                                         int max_waves) {
  const int lane = threadIdx.x & 31;
  const int vmask = W.vcap - 1;
  const int BV = FWD ? -1 : I32MAX;
  int *NA = W.NA;
  RegWave R;
  R.V = BV;
  R.M = R.HA = R.HM = R.NA = 0;
  R.T = 0;
  bool regmode = false;
  RegCtx X{vmask, W.NA, W.pool.cells, W.pool.next, W.pool.cap, W.chunk_next, W.chunk_end, 0};
  int nwaves = 0, ncells = 0, lwaves = 0;
  // the register waves' read-only inputs, held in this loop's registers
  const AlignSpec rspec = spec;
  const Seq rA = A, rB = B;
  // back to WarpWork: the pebble chunk, counts and errors
  auto sync = [&]() {
    W.chunk_next = X.chunk_next;
    W.chunk_end = X.chunk_end;
    W.err |= X.err;
    W.waves += nwaves;
    W.cells += ncells;
    nwaves = ncells = 0;
    X.err = 0;
  };
  while (more && (FWD ? lasta >= besta - TRIM_MLAG : lasta <= besta + TRIM_MLAG)) {
    if (dif > max_waves) {
      X.err |= ALN_ERR_VCAP;
      sync();
      return 1;
    }
    const int plow = low, phgh = hgh;
    low -= 1;
    hgh += 1;
    if (hgh - low + 3 > vmask + 1) {
      X.err |= ALN_ERR_VCAP;
      sync();
      return 1;
    }
    const bool grow_lo = low >= minp, grow_hi = hgh <= maxp;
    if (!grow_lo) low += 1;
    if (!grow_hi) hgh -= 1;
    const bool use_reg = phgh >= plow && hgh - low + 1 <= 32;
    nwaves += 1;
    if (W.long_waves > 0 && !W.flagged && ++lwaves >= W.long_waves) {
      // a long call: the other warps of this SM take no new task, so that it
      // runs with the SM to itself once their current tasks end
      if (lane == 0) {
        unsigned sm;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
        if (sm < SM_FLAGS) atomicExch(&W.smflag[sm], 1u);
      }
      W.flagged = 1;
    }
    ncells += hgh >= low ? hgh - low + 1 : 0;
    WaveSlice WS;
    if (use_reg) {
      if (!regmode) {
        reg_load(W, cur, plow, phgh, R);
        regmode = true;
      }
      dif += 1;
      if (reg_wave(FWD, X, rspec, rA, rB, low, hgh, plow, phgh, dif, R, besta, bestx, lasta, trima, trimx, trimd,
                        trimha, more, aclip, bclip, WS)) {
        sync();
        return 1;
      }
    } else {
      sync();
      if (regmode) {
        reg_store(W, cur, plow, phgh, R);
        regmode = false;
        __syncwarp();
      }
      // boundary diagonals on the previous wave's buffer (lane 0; visible
      // after syncwarp); the diagonal past the top carries T = PATH_INT,
      // M = PATH_LEN, HA = -1
      int *Vo = W.V[cur];
      if (lane == 0) {
        if (grow_lo) {
          NA[low & vmask] = NA[(low + 1) & vmask];
          Vo[low & vmask] = BV;
        }
        if (grow_hi) {
          NA[hgh & vmask] = NA[(hgh - 1) & vmask];
          Vo[hgh & vmask] = BV;
        }
        Vo[(hgh + 1) & vmask] = BV;
        Vo[(low - 1) & vmask] = BV;
      }
      dif += 1;
      __syncwarp();
      if (wave_sweep(FWD, W, spec, A, B, low, hgh, dif, cur, besta, bestx, lasta, trima, trimx, trimd, trimha, more,
                          aclip, bclip, WS))
        return 1;
      X.chunk_next = W.chunk_next;
      X.chunk_end = W.chunk_end;
      cur ^= 1;
      __syncwarp();
    }
    if (more == 0) {
      if (bseq[besta - bestx] != 4 && aseq[bestx] != 4) more = 1;
      // state of a diagonal of the wave just made
      auto at = [&](int kq, int &vq, int &mq, int &haq) {
        if (regmode) {
          vq = __shfl_sync(FULL, R.V, kq & 31);
          mq = __shfl_sync(FULL, R.M, kq & 31);
          haq = __shfl_sync(FULL, R.HA, kq & 31);
        } else {
          vq = W.V[cur][kq & vmask];
          mq = W.M[cur][kq & vmask];
          haq = W.HA[cur][kq & vmask];
        }
      };
      // FWD: the top side meets A's end (aclip), the bottom B's (bclip);
      // reverse: the bottom meets A's start, the top B's
      const bool cut_a = FWD ? hgh >= aclip : low <= aclip;
      if (cut_a) {
        if (FWD) hgh = aclip - 1;
        else low = aclip + 1;
        int vq, mq, haq;
        at(aclip, vq, mq, haq);
        if (morem <= mq) {
          morem = mq;
          morea = vq;
          morex = (morea + aclip) >> 1;
          mored = dif;
          moreha = haq;
        }
      }
      const bool cut_b = FWD ? low <= bclip : hgh >= bclip;
      if (cut_b) {
        if (FWD) low = bclip + 1;
        else hgh = bclip - 1;
        int vq, mq, haq;
        at(bclip, vq, mq, haq);
        if (morem <= mq) {
          morem = mq;
          morea = vq;
          morex = (morea + bclip) >> 1;
          mored = dif;
          moreha = haq;
        }
      }
      aclip = FWD ? I32MAX : -I32MAX;
      bclip = FWD ? -I32MAX : I32MAX;
    }
    if (regmode) {
      // WAVE_LAG pruning of a register wave: its one diagonal per lane
      if (hgh >= low) {
        const int n = FWD ? besta - WAVE_LAG : besta + WAVE_LAG;
        const bool pass = WS.nact && WS.k0 >= low && WS.k0 <= hgh && (FWD ? WS.c[0] >= n : WS.c[0] <= n);
        const int kmax = __reduce_max_sync(FULL, pass ? WS.k0 : -2147483647);
        const int kmin = __reduce_min_sync(FULL, pass ? WS.k0 : 2147483647);
        if (kmin <= kmax) {
          hgh = kmax;
          low = kmin;
        } else
          hgh = low - 1;
      }
    } else
      wave_prune(FWD, W, W.V[cur], besta, low, hgh, WS);
  }
  sync();
  __syncwarp();
  return 0;
}

// The wave loop's state across the call below.
struct WaveState {
  int low, hgh, dif, cur, besta, bestx, lasta, trima, trimx, trimd, trimha, more, aclip, bclip, morem, morea, morex,
      mored, moreha;
};

// One out-of-line copy of the wave loop serves both directions (FWD is a
// run-time flag).  The alignment kernel is bound by instruction fetch: two
// inlined copies of this loop, one per direction, kept twice the hot code in
// the instruction cache; one shared copy cut the pair phase of a 2 x 1 Gbp
// genome pair by a quarter with the same alignments.
__device__ __noinline__ int wave_loop_shared(const bool FWD, WarpWork &W, const AlignSpec &spec, const Seq &A,
                                             const Seq &B, const uint8_t *aseq, const uint8_t *bseq, int minp,
                                             int maxp, WaveState *io, int max_waves) {
  WaveState s = *io;
  const int r = wave_loop(FWD, W, spec, A, B, aseq, bseq, minp, maxp, s.low, s.hgh, s.dif, s.cur, s.besta, s.bestx,
                          s.lasta, s.trima, s.trimx, s.trimd, s.trimha, s.more, s.aclip, s.bclip, s.morem, s.morea,
                          s.morex, s.mored, s.moreha, max_waves);
  *io = s;
  return r;
}

// wave_loop through the shared copy, with the caller's variables.
__device__ __forceinline__ int wave_loop_call(const bool FWD, WarpWork &W, const AlignSpec &spec, const Seq &A,
                                              const Seq &B, const uint8_t *aseq, const uint8_t *bseq, int minp,
                                              int maxp, int &low, int &hgh, int &dif, int &cur, int &besta,
                                              int &bestx, int &lasta, int &trima, int &trimx, int &trimd,
                                              int &trimha, int &more, int &aclip, int &bclip, int &morem, int &morea,
                                              int &morex, int &mored, int &moreha, int max_waves) {
  WaveState s{low,   hgh,  dif,   cur,   besta, bestx, lasta, trima, trimx, trimd,
              trimha, more, aclip, bclip, morem, morea, morex, mored, moreha};
  const int r = wave_loop_shared(FWD, W, spec, A, B, aseq, bseq, minp, maxp, &s, max_waves);
  low = s.low, hgh = s.hgh, dif = s.dif, cur = s.cur, besta = s.besta, bestx = s.bestx, lasta = s.lasta;
  trima = s.trima, trimx = s.trimx, trimd = s.trimd, trimha = s.trimha, more = s.more, aclip = s.aclip;
  bclip = s.bclip, morem = s.morem, morea = s.morea, morex = s.morex, mored = s.mored, moreha = s.moreha;
  return r;
}

#define WVI(k) ((k) & vmask)

// ---------------------------------------------------------------------------
// forward_wave, warp version.  Returns 1 on an arena overflow (W.err set).
// ---------------------------------------------------------------------------
__device__ int forward_wave_w(WarpWork &W, const AlignSpec &spec, const Seq &A, const Seq &B, Path &P, int *mind,
                              int maxd, int mida, int minp, int maxp, int aoff) {
  const int lane = threadIdx.x & 31;
  const uint8_t *aseq = A.s;
  const uint8_t *bseq = B.s;
  const int vmask = W.vcap - 1;
  int cur = 0;
  int *NA = W.NA;
  Pebble *cells = W.pool.cells;
  const int tspace = spec.trace_space;

  int hgh = maxd, low = *mind, dif = 0;
  int besta, bestx, trima, trimx, trimd, trimha, morea, morex, mored, moreha, more, morem, lasta;
  int aclip, bclip;
  if (hgh - low + 3 > W.vcap) {
    W.err |= ALN_ERR_VCAP;
    return 1;
  }
  more = 1;
  aclip = I32MAX;
  bclip = -I32MAX;
  besta = trima = morea = lasta = mida;
  bestx = trimx = morex = (mida + hgh) >> 1;
  trimd = mored = 0;
  trimha = moreha = 0;
  morem = -1;
  int64_t call_base = -1;  // this call's first pebble: the reference's cells[0]
  const int max_waves = A.len + B.len + 1024;

  // 0-wave: diagonals visited hgh..low
  for (int base = hgh; base >= low; base -= 32) {
    int k = base - lane;
    bool act = k >= low;
    int x = 0, c = 0, na = 0, hb = 0, ha_ = 0, npb = 0;
    if (act) {
      x = (mida + k) >> 1;
      na = ((x + (tspace - aoff)) / tspace - 1) * tspace + aoff;
      x = snake_fwd(A, B, x, k, &hb, &ha_);
      c = (x << 1) - k;
      npb = 1;
      for (int q = na + tspace; x >= q; q += tspace) npb++;
    }
    int off = warp_excl_sum(npb, lane);
    int tot = warp_sum(npb);
    int64_t pb0 = warp_pebbles(W, tot);
    if (pb0 < 0) return 1;
    if (call_base < 0) {
      call_base = pb0;
      trimha = moreha = (int)pb0;
    }
    int ha = -1;
    if (act) {
      int64_t s = pb0 + off;
      cells[s] = {-1, k, 0, na};
      ha = (int)s;
      int hm = na;
      na += tspace;
      while (x >= na) {
        s += 1;
        cells[s] = {ha, k, 0, na};
        ha = (int)s;
        hm = na;
        na += tspace;
      }
      int vi = WVI(k);
      W.V[cur][vi] = c;
      W.T[cur][vi] = PATH_INT;
      W.M[cur][vi] = PATH_LEN;
      W.HA[cur][vi] = ha;
      W.HM[cur][vi] = hm;
      NA[vi] = na;
    }
    // clips: bclip = largest k that met B's end, aclip = last visited (smallest) k that met A's end
    uint32_t bb = __ballot_sync(FULL, act && hb), ba = __ballot_sync(FULL, act && ha_);
    if (bb) {
      more = 0;
      int kk = base - (__ffs(bb) - 1);
      if (bclip < kk) bclip = kk;
    }
    if (ba) {
      more = 0;
      aclip = base - last_lane(ba);
    }
    // records: c > running maximum
    int pm = warp_excl_max(act ? c : -2147483647, lane, besta);
    bool rec = act && c > pm;
    uint32_t rb = __ballot_sync(FULL, rec);
    if (rb) {
      int L = last_lane(rb);
      besta = trima = lasta = __shfl_sync(FULL, c, L);
      bestx = trimx = __shfl_sync(FULL, x, L);
      trimha = __shfl_sync(FULL, ha, L);
    }
  }
  __syncwarp();
  {
    int *V = W.V[cur], *M = W.M[cur], *HA = W.HA[cur];
    if (more == 0) {
      if (bseq[besta - bestx] != 4 && aseq[bestx] != 4) more = 1;
      if (hgh >= aclip) {
        hgh = aclip - 1;
        if (morem <= M[WVI(aclip)]) {
          morem = M[WVI(aclip)];
          morea = V[WVI(aclip)];
          morex = (morea + aclip) >> 1;
          moreha = HA[WVI(aclip)];
        }
      }
      if (low <= bclip) {
        low = bclip + 1;
        if (morem <= M[WVI(bclip)]) {
          morem = M[WVI(bclip)];
          morea = V[WVI(bclip)];
          morex = (morea + bclip) >> 1;
          moreha = HA[WVI(bclip)];
        }
      }
      aclip = I32MAX;
      bclip = -I32MAX;
    }
  }

  if (wave_loop_call(true, W, spec, A, B, aseq, bseq, minp, maxp, low, hgh, dif, cur, besta, bestx, lasta, trima,
                     trimx, trimd, trimha, more, aclip, bclip, morem, morea, morex, mored, moreha, max_waves))
    return 1;
  __syncwarp();

  // trace-back (lane-uniform sequential code; only lane 0 writes)
  {
    uint16_t *atrace = W.points + P.trace_off;
    int atlen = 0, trimy, a, b, k, h, d, e;
    if (morem >= 0 && spec.reach) {
      trimx = morex;
      trimy = morea - morex;
      trimd = mored;
      trimha = moreha;
    } else
      trimy = trima - trimx;
    // reverse the pebble chain: done by lane 0, read back by all
    int bad = 0;
    if (lane == 0) {
      int64_t steps = 0, lim = W.chunk_next - call_base + 1;
      a = -1;
      for (h = trimha; h >= 0; h = b) {
        if (h < call_base || ++steps > lim) {
          bad = 1;
          break;
        }
        b = cells[h].ptr;
        cells[h].ptr = a;
        a = h;
      }
    }
    if (__shfl_sync(FULL, bad, 0)) {
      W.err |= ALN_ERR_CELLS;
      return 1;
    }
    __syncwarp();
    a = __shfl_sync(FULL, a, 0);
    h = a;
    k = cells[h].diag;
    b = (mida - k) >> 1;
    e = 0;
    low = k;
    for (h = cells[h].ptr; h >= 0; h = cells[h].ptr) {
      k = cells[h].diag;
      a = cells[h].mark - k;
      d = cells[h].diff;
      if (P.trace_off + atlen + 2 > W.point_cap) {
        W.err |= ALN_ERR_POINTS;
        return 1;
      }
      if (lane == 0) {
        atrace[atlen] = (uint16_t)(d - e);
        atrace[atlen + 1] = (uint16_t)(a - b);
      }
      atlen += 2;
      b = a;
      e = d;
    }
    __syncwarp();
    if (b + k != trimx) {
      if (P.trace_off + atlen + 2 > W.point_cap) {
        W.err |= ALN_ERR_POINTS;
        return 1;
      }
      if (lane == 0) {
        atrace[atlen] = (uint16_t)(trimd - e);
        atrace[atlen + 1] = (uint16_t)(trimy - b);
      }
      atlen += 2;
    } else if (b != trimy) {
      if (lane == 0) {
        atrace[atlen - 1] = (uint16_t)(atrace[atlen - 1] + (trimy - b));
        atrace[atlen - 2] = (uint16_t)(atrace[atlen - 2] + (trimd - e));
      }
    }
    __syncwarp();
    P.aepos = trimx;
    P.bepos = trimy;
    P.diffs = trimd;
    P.tlen = atlen;
  }
  *mind = low;
  return 0;
}

// ---------------------------------------------------------------------------
// reverse_wave, warp version (visit order k = low..hgh, minimum instead of
// maximum, sequences read one position to the left).
// ---------------------------------------------------------------------------
__device__ int reverse_wave_w(WarpWork &W, const AlignSpec &spec, const Seq &A, const Seq &B, Path &P, int mind,
                              int maxd, int mida, int minp, int maxp, int aoff) {
  const int lane = threadIdx.x & 31;
  const uint8_t *aseq = A.s - 1;
  const uint8_t *bseq = B.s - 1;
  const int vmask = W.vcap - 1;
  int cur = 0;
  int *NA = W.NA;
  Pebble *cells = W.pool.cells;
  const int tspace = spec.trace_space;

  int hgh = maxd, low = mind, dif = 0;
  int besta, bestx, trima, trimx, trimd, trimha, morea, morex, mored, moreha, more, morem, lasta;
  int aclip, bclip;
  if (hgh - low + 3 > W.vcap) {
    W.err |= ALN_ERR_VCAP;
    return 1;
  }
  more = 1;
  aclip = -I32MAX;
  bclip = I32MAX;
  besta = trima = morea = lasta = mida;
  bestx = trimx = morex = (mida + hgh) >> 1;
  trimd = mored = 0;
  trimha = moreha = 0;
  morem = -1;
  int64_t call_base = -1;  // this call's first pebble: the reference's cells[0]
  const int max_waves = A.len + B.len + 1024;

  for (int base = low; base <= hgh; base += 32) {
    int k = base + lane;
    bool act = k <= hgh;
    int x = 0, c = 0, na = 0, hb = 0, hA = 0, npb = 0, x0 = 0;
    if (act) {
      x = (mida + k) >> 1;
      x0 = x;
      na = ((x + (tspace - aoff) - 1) / tspace - 1) * tspace + aoff;
      x = snake_rev(A, B, x, k, &hb, &hA);
      c = (x << 1) - k;
      npb = 1;
      for (int q = na; x <= q; q -= tspace) npb++;
    }
    int off = warp_excl_sum(npb, lane);
    int tot = warp_sum(npb);
    int64_t pb0 = warp_pebbles(W, tot);
    if (pb0 < 0) return 1;
    if (call_base < 0) {
      call_base = pb0;
      trimha = moreha = (int)pb0;
    }
    int ha = -1;
    if (act) {
      int64_t s = pb0 + off;
      cells[s] = {-1, k, 0, x0};
      ha = (int)s;
      int hm = x0;
      while (x <= na) {
        s += 1;
        cells[s] = {ha, k, 0, na};
        ha = (int)s;
        hm = na;
        na -= tspace;
      }
      int vi = WVI(k);
      W.V[cur][vi] = c;
      W.T[cur][vi] = PATH_INT;
      W.M[cur][vi] = PATH_LEN;
      W.HA[cur][vi] = ha;
      W.HM[cur][vi] = hm;
      NA[vi] = na;
    }
    // bclip = smallest k that met B's start, aclip = last visited (largest) k that met A's start
    uint32_t bb = __ballot_sync(FULL, act && hb), ba = __ballot_sync(FULL, act && hA);
    if (bb) {
      more = 0;
      int kk = base + (__ffs(bb) - 1);
      if (bclip > kk) bclip = kk;
    }
    if (ba) {
      more = 0;
      aclip = base + last_lane(ba);
    }
    int pm = warp_excl_min(act ? c : 2147483647, lane, besta);
    bool rec = act && c < pm;
    uint32_t rb = __ballot_sync(FULL, rec);
    if (rb) {
      int L = last_lane(rb);
      besta = trima = lasta = __shfl_sync(FULL, c, L);
      bestx = trimx = __shfl_sync(FULL, x, L);
      trimha = __shfl_sync(FULL, ha, L);
    }
  }
  __syncwarp();
  {
    int *V = W.V[cur], *M = W.M[cur], *HA = W.HA[cur];
    if (more == 0) {
      if (bseq[besta - bestx] != 4 && aseq[bestx] != 4) more = 1;
      if (low <= aclip) {
        low = aclip + 1;
        if (morem <= M[WVI(aclip)]) {
          morem = M[WVI(aclip)];
          morea = V[WVI(aclip)];
          morex = (morea + aclip) >> 1;
          moreha = HA[WVI(aclip)];
        }
      }
      if (hgh >= bclip) {
        hgh = bclip - 1;
        if (morem <= M[WVI(bclip)]) {
          morem = M[WVI(bclip)];
          morea = V[WVI(bclip)];
          morex = (morea + bclip) >> 1;
          moreha = HA[WVI(bclip)];
        }
      }
      aclip = -I32MAX;
      bclip = I32MAX;
    }
  }

  if (wave_loop_call(false, W, spec, A, B, aseq, bseq, minp, maxp, low, hgh, dif, cur, besta, bestx, lasta, trima,
                     trimx, trimd, trimha, more, aclip, bclip, morem, morea, morex, mored, moreha, max_waves))
    return 1;
  __syncwarp();

  {
    uint16_t *atrace = W.points + P.trace_off;
    int atlen = 0, trimy, a, b, k, h, d, e;
    if (morem >= 0 && spec.reach) {
      trimx = morex;
      trimy = morea - morex;
      trimd = mored;
      trimha = moreha;
    } else
      trimy = trima - trimx;
    int bad = 0;
    if (lane == 0) {
      int64_t steps = 0, lim = W.chunk_next - call_base + 1;
      a = -1;
      for (h = trimha; h >= 0; h = b) {
        if (h < call_base || ++steps > lim) {
          bad = 1;
          break;
        }
        b = cells[h].ptr;
        cells[h].ptr = a;
        a = h;
      }
    }
    if (__shfl_sync(FULL, bad, 0)) {
      W.err |= ALN_ERR_CELLS;
      return 1;
    }
    __syncwarp();
    a = __shfl_sync(FULL, a, 0);
    h = a;
    k = cells[h].diag;
    b = cells[h].mark - k;
    e = 0;
    if ((b + k) % tspace != aoff) {
      h = cells[h].ptr;
      if (h < 0) {
        a = trimy;
        d = trimd;
      } else {
        k = cells[h].diag;
        a = cells[h].mark - k;
        d = cells[h].diff;
      }
      if (P.tlen == 0) {
        if (P.trace_off + atlen - 2 < 0) {
          W.err |= ALN_ERR_POINTS;
          return 1;
        }
        if (lane == 0) {
          atrace[atlen - 1] = (uint16_t)(b - a);
          atrace[atlen - 2] = (uint16_t)(d - e);
        }
        atlen -= 2;
      } else if (lane == 0) {
        atrace[1] = (uint16_t)(atrace[1] + (b - a));
        atrace[0] = (uint16_t)(atrace[0] + (d - e));
      }
      b = a;
      e = d;
    }
    if (h >= 0) {
      for (h = cells[h].ptr; h >= 0; h = cells[h].ptr) {
        k = cells[h].diag;
        a = cells[h].mark - k;
        if (P.trace_off + atlen - 2 < 0) {
          W.err |= ALN_ERR_POINTS;
          return 1;
        }
        d = cells[h].diff;
        if (lane == 0) {
          atrace[atlen - 1] = (uint16_t)(b - a);
          atrace[atlen - 2] = (uint16_t)(d - e);
        }
        atlen -= 2;
        b = a;
        e = d;
      }
      __syncwarp();
      if (b + k != trimx) {
        if (P.trace_off + atlen - 2 < 0) {
          W.err |= ALN_ERR_POINTS;
          return 1;
        }
        if (lane == 0) {
          atrace[atlen - 1] = (uint16_t)(b - trimy);
          atrace[atlen - 2] = (uint16_t)(trimd - e);
        }
        atlen -= 2;
      } else if (b != trimy) {
        if (lane == 0) {
          atrace[atlen + 1] = (uint16_t)(atrace[atlen + 1] + (b - trimy));
          atrace[atlen] = (uint16_t)(atrace[atlen] + (trimd - e));
        }
      }
    }
    __syncwarp();
    P.abpos = trimx;
    P.bbpos = trimy;
    P.diffs = P.diffs + trimd;
    P.tlen = P.tlen - atlen;
    P.trace_off = P.trace_off + atlen;
  }
  return 0;
}

#undef WVI

// A path on the complemented A (and so on reversed B coordinates) in
// forward coordinates: both intervals mirrored, and the trace-point pairs
// (diffs, b-delta) in the opposite order, the warp's lanes swapping pair q
// with pair npairs-1-q.
__device__ __forceinline__ void path_to_forward(uint16_t *trace, const Seq &A, const Seq &B, Path &P) {
  const int lane = threadIdx.x & 31;
  const int ab = P.abpos, bb = P.bbpos;
  P.abpos = A.len - P.aepos;
  P.aepos = A.len - ab;
  P.bbpos = B.len - P.bepos;
  P.bepos = B.len - bb;
  const int npairs = P.tlen >> 1;
  __syncwarp();
  for (int q = lane; q < npairs / 2; q += 32) {
    uint32_t *x = reinterpret_cast<uint32_t *>(trace) + q, *y = reinterpret_cast<uint32_t *>(trace) + (npairs - 1 - q);
    const uint32_t t = *x;
    *x = *y;
    *y = t;
  }
  __syncwarp();
}

// Local_Alignment (lib/align.c:1423-1576) on one warp.  The path is grown
// forward from the seed point (antidiagonal `anti`, diagonals [low, hgh],
// kept within `lbord` / `hbord` of them when those are set), then backward
// from the diagonal the forward pass started on.  An end that moved fewer
// than DUB_TRIM antidiagonals from `anti` did not get away from the seed:
// with both ends short the path shrinks to the midpoint of the two, without
// trace points; with one end short, that direction runs again from the end
// the other direction reached (a forward re-run keeps the reverse pass's
// start, a reverse re-run counts its differences afresh).  With `acomp` A is
// the complemented contig and the path comes back in forward coordinates.
// Returns 1 on a work-space overflow (W.err says which).
__device__ __forceinline__ int local_alignment_w(WarpWork &W, const AlignSpec &spec, const Seq &A, const Seq &B,
                                                 bool acomp, Path &P, int low, int hgh, int anti, int lbord,
                                                 int hbord) {
  const int maxtp = 2 * (A.len / spec.trace_space + 2);  // trace points the longest path can have
  if (2 * (int64_t)maxtp > W.point_cap) {
    W.err |= ALN_ERR_POINTS;
    return 1;
  }
  P.trace_off = maxtp;
  while (((anti - hgh) >> 1) < 0) hgh -= 1;  // no diagonal above the antidiagonal's start
  const int minp = lbord < 0 ? -I32MAX : low - lbord;
  const int maxp = hbord < 0 ? I32MAX : hgh + hbord;
  const int aoff = acomp ? A.len % spec.trace_space : 0;

  if (forward_wave_w(W, spec, A, B, P, &low, hgh, anti, minp, maxp, aoff)) return 1;
  const bool fwd_away = (P.aepos + P.bepos) - anti >= DUB_TRIM;
  if (reverse_wave_w(W, spec, A, B, P, low, low, anti, minp, maxp, aoff)) return 1;
  const bool rev_away = anti - (P.abpos + P.bbpos) >= DUB_TRIM;

  if (!fwd_away && !rev_away) {
    P.aepos = P.abpos = (P.abpos + P.aepos) >> 1;
    P.bepos = P.bbpos = (P.bbpos + P.bepos) >> 1;
    P.tlen = 0;
  } else if (!fwd_away) {
    int from = P.abpos - P.bbpos;
    P.tlen = 0;
    if (forward_wave_w(W, spec, A, B, P, &from, from, P.abpos + P.bbpos, minp, maxp, aoff)) return 1;
  } else if (!rev_away) {
    const int from = P.aepos - P.bepos, at = P.aepos + P.bepos;
    P.tlen = 0;
    P.diffs = 0;
    if (reverse_wave_w(W, spec, A, B, P, from, from, at, minp, maxp, aoff)) return 1;
  }
  if (acomp) path_to_forward(W.points + P.trace_off, A, B, P);
  return 0;
}

}  // namespace aln
}  // namespace pga
