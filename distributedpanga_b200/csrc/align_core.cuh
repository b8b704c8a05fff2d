// FastGA's wave aligner and chain driver, as scalar code shared by the host
// (tests, CPU reruns) and the device.
//
// Restates, for one (anchor, partner) contig pair:
//   forward_wave / reverse_wave / Local_Alignment   lib/align.c:352-1576
//   align_contigs (chaining, window calls, filter,
//     sort, duplicate / containment elimination,
//     entwine merge, box elimination)               src/fastga_pipeline.c:505-993
//   Compress_TraceTo8                               lib/align.c:3892-3910
//
// Differences of representation only: per-diagonal wave vectors live in ring
// buffers indexed by diagonal & (vcap - 1) instead of a re-centred window (the
// values are the same; a band wider than vcap - 2 diagonals sets ALN_ERR_VCAP),
// trace-point pebbles and trace points live in caller-provided arenas of fixed
// capacity (overflow sets an error bit so the caller can rerun the pair with
// more room), and seeds are read from decoded fields instead of swide bytes.
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
  int trace_off;  // start of the trace (uint16 pairs) in WaveWork::points
};

// Per-worker scratch for the waves of one Local_Alignment call.
struct WaveWork {
  int *V, *M, *HA, *NA;
  uint64_t *T;
  int vcap;            // power of two
  Pebble *cells;
  int64_t cell_cap;
  uint16_t *points;    // trace points; a call uses 2*maxtp entries
  int64_t point_cap;
  int err;
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

#define PGA_VI(k) ((k) & vmask)

// ---------------------------------------------------------------------------
// forward_wave (lib/align.c:352-874)
// ---------------------------------------------------------------------------
PGA_HD int forward_wave(WaveWork &W, const AlignSpec &spec, const Seq &A, const Seq &B, Path &P,
                        int *mind, int maxd, int mida, int minp, int maxp, int aoff) {
  const uint8_t *aseq = A.s;
  const uint8_t *bseq = B.s;
  const int vmask = W.vcap - 1;
  int *V = W.V, *M = W.M, *HA = W.HA, *NA = W.NA;
  uint64_t *T = W.T;
  Pebble *cells = W.cells;
  const int64_t cmax = W.cell_cap;
  int64_t avail = 0;
  const int tspace = spec.trace_space;
  const int PATH_AVE = spec.ave_path;
  const int REACH = spec.reach;
  const int16_t *SCORE = spec.score;
  const int16_t *TABLE = spec.table;

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

  // 0-wave from the mid-line (lib/align.c:428-509)
  for (int k = hgh; k >= low; k--) {
    int x, c, d, ha, na;
    x = (mida + k) >> 1;
    if (avail >= cmax - 1) {
      W.err |= ALN_ERR_CELLS;
      return 1;
    }
    na = ((x + (tspace - aoff)) / tspace - 1) * tspace + aoff;
    cells[avail] = {-1, k, 0, na};
    ha = (int)avail++;
    na += tspace;
    while (1) {
      c = bseq[x - k];
      if (c == 4) {
        more = 0;
        if (bclip < k) bclip = k;
        break;
      }
      d = aseq[x];
      if (c != d) {
        if (d == 4) {
          more = 0;
          aclip = k;
        }
        break;
      }
      x += 1;
    }
    c = (x << 1) - k;
    while (x >= na) {
      if (avail >= cmax) {
        W.err |= ALN_ERR_CELLS;
        return 1;
      }
      cells[avail] = {ha, k, 0, na};
      ha = (int)avail++;
      na += tspace;
    }
    if (c > besta) {
      besta = trima = lasta = c;
      bestx = trimx = x;
      trimha = ha;
    }
    V[PGA_VI(k)] = c;
    T[PGA_VI(k)] = PATH_INT;
    M[PGA_VI(k)] = PATH_LEN;
    HA[PGA_VI(k)] = ha;
    NA[PGA_VI(k)] = na;
  }

  if (more == 0) {
    if (bseq[besta - bestx] != 4 && aseq[bestx] != 4) more = 1;
    if (hgh >= aclip) {
      hgh = aclip - 1;
      if (morem <= M[PGA_VI(aclip)]) {
        morem = M[PGA_VI(aclip)];
        morea = V[PGA_VI(aclip)];
        morex = (morea + aclip) >> 1;
        moreha = HA[PGA_VI(aclip)];
      }
    }
    if (low <= bclip) {
      low = bclip + 1;
      if (morem <= M[PGA_VI(bclip)]) {
        morem = M[PGA_VI(bclip)];
        morea = V[PGA_VI(bclip)];
        morex = (morea + bclip) >> 1;
        moreha = HA[PGA_VI(bclip)];
      }
    }
    aclip = I32MAX;
    bclip = -I32MAX;
  }

  // successive waves (lib/align.c:541-781)
  while (more && lasta >= besta - TRIM_MLAG) {
    int k, n, ua, am, ac, ap;
    uint64_t t;
    low -= 1;
    hgh += 1;
    if (hgh - low + 3 > W.vcap) {
      W.err |= ALN_ERR_VCAP;
      return 1;
    }
    if (low >= minp) {
      NA[PGA_VI(low)] = NA[PGA_VI(low + 1)];
      V[PGA_VI(low)] = -1;
    } else
      low += 1;
    if (hgh <= maxp) {
      NA[PGA_VI(hgh)] = NA[PGA_VI(hgh - 1)];
      V[PGA_VI(hgh)] = am = -1;
    } else
      am = V[PGA_VI(--hgh)];
    dif += 1;
    ac = V[PGA_VI(hgh + 1)] = V[PGA_VI(low - 1)] = -1;
    t = PATH_INT;
    n = PATH_LEN;
    ua = -1;
    for (k = hgh; k >= low; k--) {
      int x, m, ha, c, d;
      uint64_t b;
      ap = ac;
      ac = am;
      am = V[PGA_VI(d = k - 1)];
      if (ac < am)
        if (am < ap) {
          c = ap + 1; m = n; b = t; ha = ua;
        } else {
          c = am + 1; m = M[PGA_VI(d)]; b = T[PGA_VI(d)]; ha = HA[PGA_VI(d)];
        }
      else if (ac < ap) {
        c = ap + 1; m = n; b = t; ha = ua;
      } else {
        c = ac + 2; m = M[PGA_VI(k)]; b = T[PGA_VI(k)]; ha = HA[PGA_VI(k)];
      }
      if ((b & PATH_TOP) != 0) m -= 1;
      b <<= 1;
      x = (c + k) >> 1;
      while (1) {
        c = bseq[x - k];
        if (c == 4) {
          more = 0;
          if (bclip < k) bclip = k;
          break;
        }
        d = aseq[x];
        if (c != d) {
          if (d == 4) {
            more = 0;
            aclip = k;
          }
          break;
        }
        x += 1;
        if ((b & PATH_TOP) == 0) m += 1;
        b = (b << 1) | 1;
      }
      c = (x << 1) - k;
      while (x >= NA[PGA_VI(k)]) {
        if (cells[ha].mark < NA[PGA_VI(k)]) {
          if (avail >= cmax) {
            W.err |= ALN_ERR_CELLS;
            return 1;
          }
          cells[avail] = {ha, k, dif, NA[PGA_VI(k)]};
          ha = (int)avail++;
        }
        NA[PGA_VI(k)] += tspace;
      }
      if (c > besta) {
        besta = c;
        bestx = x;
        if (m >= PATH_AVE) {
          lasta = c;
          if (TABLE[b & TRIM_MASK] >= 0)
            if (TABLE[(b >> TRIM_LEN) & TRIM_MASK] + SCORE[b & TRIM_MASK] >= 0) {
              trima = c; trimx = x; trimd = dif; trimha = ha;
            }
        }
      }
      t = T[PGA_VI(k)];
      n = M[PGA_VI(k)];
      ua = HA[PGA_VI(k)];
      V[PGA_VI(k)] = c;
      T[PGA_VI(k)] = b;
      M[PGA_VI(k)] = m;
      HA[PGA_VI(k)] = ha;
    }
    if (more == 0) {
      if (bseq[besta - bestx] != 4 && aseq[bestx] != 4) more = 1;
      if (hgh >= aclip) {
        hgh = aclip - 1;
        if (morem <= M[PGA_VI(aclip)]) {
          morem = M[PGA_VI(aclip)];
          morea = V[PGA_VI(aclip)];
          morex = (morea + aclip) >> 1;
          mored = dif;
          moreha = HA[PGA_VI(aclip)];
        }
      }
      if (low <= bclip) {
        low = bclip + 1;
        if (morem <= M[PGA_VI(bclip)]) {
          morem = M[PGA_VI(bclip)];
          morea = V[PGA_VI(bclip)];
          morex = (morea + bclip) >> 1;
          mored = dif;
          moreha = HA[PGA_VI(bclip)];
        }
      }
      aclip = I32MAX;
      bclip = -I32MAX;
    }
    n = besta - WAVE_LAG;
    while (hgh >= low)
      if (V[PGA_VI(hgh)] < n)
        hgh -= 1;
      else {
        while (V[PGA_VI(low)] < n) low += 1;
        break;
      }
  }

  // trace points of the forward half (lib/align.c:806-871)
  {
    uint16_t *atrace = W.points + P.trace_off;
    int atlen = 0, trimy, a, b, k, h, d, e;
    if (morem >= 0 && REACH) {
      trimx = morex;
      trimy = morea - morex;
      trimd = mored;
      trimha = moreha;
    } else
      trimy = trima - trimx;
    a = -1;
    for (h = trimha; h >= 0; h = b) {
      b = cells[h].ptr;
      cells[h].ptr = a;
      a = h;
    }
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
      atrace[atlen++] = (uint16_t)(d - e);
      atrace[atlen++] = (uint16_t)(a - b);
      b = a;
      e = d;
    }
    if (b + k != trimx) {
      if (P.trace_off + atlen + 2 > W.point_cap) {
        W.err |= ALN_ERR_POINTS;
        return 1;
      }
      atrace[atlen++] = (uint16_t)(trimd - e);
      atrace[atlen++] = (uint16_t)(trimy - b);
    } else if (b != trimy) {
      atrace[atlen - 1] = (uint16_t)(atrace[atlen - 1] + (trimy - b));
      atrace[atlen - 2] = (uint16_t)(atrace[atlen - 2] + (trimd - e));
    }
    P.aepos = trimx;
    P.bepos = trimy;
    P.diffs = trimd;
    P.tlen = atlen;
  }
  *mind = low;
  return 0;
}

// ---------------------------------------------------------------------------
// reverse_wave (lib/align.c:878-1421); sequences are read one position to the
// left (aseq = A - 1, bseq = B - 1) as in the reference.
// ---------------------------------------------------------------------------
PGA_HD int reverse_wave(WaveWork &W, const AlignSpec &spec, const Seq &A, const Seq &B, Path &P,
                        int mind, int maxd, int mida, int minp, int maxp, int aoff) {
  const uint8_t *aseq = A.s - 1;
  const uint8_t *bseq = B.s - 1;
  const int vmask = W.vcap - 1;
  int *V = W.V, *M = W.M, *HA = W.HA, *NA = W.NA;
  uint64_t *T = W.T;
  Pebble *cells = W.cells;
  const int64_t cmax = W.cell_cap;
  int64_t avail = 0;
  const int tspace = spec.trace_space;
  const int PATH_AVE = spec.ave_path;
  const int REACH = spec.reach;
  const int16_t *SCORE = spec.score;
  const int16_t *TABLE = spec.table;

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

  for (int k = low; k <= hgh; k++) {
    int x, c, d, ha, na;
    x = (mida + k) >> 1;
    if (avail >= cmax - 1) {
      W.err |= ALN_ERR_CELLS;
      return 1;
    }
    na = ((x + (tspace - aoff) - 1) / tspace - 1) * tspace + aoff;
    cells[avail] = {-1, k, 0, x};
    ha = (int)avail++;
    while (1) {
      c = bseq[x - k];
      if (c == 4) {
        more = 0;
        if (bclip > k) bclip = k;
        break;
      }
      d = aseq[x];
      if (c != d) {
        if (d == 4) {
          more = 0;
          aclip = k;
        }
        break;
      }
      x -= 1;
    }
    c = (x << 1) - k;
    while (x <= na) {
      if (avail >= cmax) {
        W.err |= ALN_ERR_CELLS;
        return 1;
      }
      cells[avail] = {ha, k, 0, na};
      ha = (int)avail++;
      na -= tspace;
    }
    if (c < besta) {
      besta = trima = lasta = c;
      bestx = trimx = x;
      trimha = ha;
    }
    V[PGA_VI(k)] = c;
    T[PGA_VI(k)] = PATH_INT;
    M[PGA_VI(k)] = PATH_LEN;
    HA[PGA_VI(k)] = ha;
    NA[PGA_VI(k)] = na;
  }

  if (more == 0) {
    if (bseq[besta - bestx] != 4 && aseq[bestx] != 4) more = 1;
    if (low <= aclip) {
      low = aclip + 1;
      if (morem <= M[PGA_VI(aclip)]) {
        morem = M[PGA_VI(aclip)];
        morea = V[PGA_VI(aclip)];
        morex = (morea + aclip) >> 1;
        moreha = HA[PGA_VI(aclip)];
      }
    }
    if (hgh >= bclip) {
      hgh = bclip - 1;
      if (morem <= M[PGA_VI(bclip)]) {
        morem = M[PGA_VI(bclip)];
        morea = V[PGA_VI(bclip)];
        morex = (morea + bclip) >> 1;
        moreha = HA[PGA_VI(bclip)];
      }
    }
    aclip = -I32MAX;
    bclip = I32MAX;
  }

  while (more && lasta <= besta + TRIM_MLAG) {
    int k, n, ua, am, ac, ap;
    uint64_t t;
    low -= 1;
    hgh += 1;
    if (hgh - low + 3 > W.vcap) {
      W.err |= ALN_ERR_VCAP;
      return 1;
    }
    if (low >= minp) {
      NA[PGA_VI(low)] = NA[PGA_VI(low + 1)];
      V[PGA_VI(low)] = ap = I32MAX;
    } else
      ap = V[PGA_VI(++low)];
    if (hgh <= maxp) {
      NA[PGA_VI(hgh)] = NA[PGA_VI(hgh - 1)];
      V[PGA_VI(hgh)] = I32MAX;
    } else
      hgh -= 1;
    dif += 1;
    ac = V[PGA_VI(hgh + 1)] = V[PGA_VI(low - 1)] = I32MAX;
    t = PATH_INT;
    n = PATH_LEN;
    ua = -1;
    for (k = low; k <= hgh; k++) {
      int x, m, ha, c, d;
      uint64_t b;
      am = ac;
      ac = ap;
      ap = V[PGA_VI(d = k + 1)];
      if (ac > ap)
        if (ap > am) {
          c = am - 1; m = n; b = t; ha = ua;
        } else {
          c = ap - 1; m = M[PGA_VI(d)]; b = T[PGA_VI(d)]; ha = HA[PGA_VI(d)];
        }
      else if (ac > am) {
        c = am - 1; m = n; b = t; ha = ua;
      } else {
        c = ac - 2; m = M[PGA_VI(k)]; b = T[PGA_VI(k)]; ha = HA[PGA_VI(k)];
      }
      if ((b & PATH_TOP) != 0) m -= 1;
      b <<= 1;
      x = (c + k) >> 1;
      while (1) {
        c = bseq[x - k];
        if (c == 4) {
          more = 0;
          if (bclip > k) bclip = k;
          break;
        }
        d = aseq[x];
        if (c != d) {
          if (d == 4) {
            more = 0;
            aclip = k;
          }
          break;
        }
        x -= 1;
        if ((b & PATH_TOP) == 0) m += 1;
        b = (b << 1) | 1;
      }
      c = (x << 1) - k;
      while (x <= NA[PGA_VI(k)]) {
        if (cells[ha].mark > NA[PGA_VI(k)]) {
          if (avail >= cmax) {
            W.err |= ALN_ERR_CELLS;
            return 1;
          }
          cells[avail] = {ha, k, dif, NA[PGA_VI(k)]};
          ha = (int)avail++;
        }
        NA[PGA_VI(k)] -= tspace;
      }
      if (c < besta) {
        besta = c;
        bestx = x;
        if (m >= PATH_AVE) {
          lasta = c;
          if (TABLE[b & TRIM_MASK] >= 0)
            if (TABLE[(b >> TRIM_LEN) & TRIM_MASK] + SCORE[b & TRIM_MASK] >= 0) {
              trima = c; trimx = x; trimd = dif; trimha = ha;
            }
        }
      }
      t = T[PGA_VI(k)];
      n = M[PGA_VI(k)];
      ua = HA[PGA_VI(k)];
      V[PGA_VI(k)] = c;
      T[PGA_VI(k)] = b;
      M[PGA_VI(k)] = m;
      HA[PGA_VI(k)] = ha;
    }
    if (more == 0) {
      if (bseq[besta - bestx] != 4 && aseq[bestx] != 4) more = 1;
      if (low <= aclip) {
        low = aclip + 1;
        if (morem <= M[PGA_VI(aclip)]) {
          morem = M[PGA_VI(aclip)];
          morea = V[PGA_VI(aclip)];
          morex = (morea + aclip) >> 1;
          mored = dif;
          moreha = HA[PGA_VI(aclip)];
        }
      }
      if (hgh >= bclip) {
        hgh = bclip - 1;
        if (morem <= M[PGA_VI(bclip)]) {
          morem = M[PGA_VI(bclip)];
          morea = V[PGA_VI(bclip)];
          morex = (morea + bclip) >> 1;
          mored = dif;
          moreha = HA[PGA_VI(bclip)];
        }
      }
      aclip = -I32MAX;
      bclip = I32MAX;
    }
    n = besta + WAVE_LAG;
    while (hgh >= low)
      if (V[PGA_VI(hgh)] > n)
        hgh -= 1;
      else {
        while (V[PGA_VI(low)] > n) low += 1;
        break;
      }
  }

  // trace points of the reverse half, prepended (lib/align.c:1323-1419)
  {
    uint16_t *atrace = W.points + P.trace_off;
    int atlen = 0, trimy, a, b, k, h, d, e;
    if (morem >= 0 && REACH) {
      trimx = morex;
      trimy = morea - morex;
      trimd = mored;
      trimha = moreha;
    } else
      trimy = trima - trimx;
    a = -1;
    for (h = trimha; h >= 0; h = b) {
      b = cells[h].ptr;
      cells[h].ptr = a;
      a = h;
    }
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
        atrace[--atlen] = (uint16_t)(b - a);
        atrace[--atlen] = (uint16_t)(d - e);
      } else {
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
        atrace[--atlen] = (uint16_t)(b - a);
        d = cells[h].diff;
        atrace[--atlen] = (uint16_t)(d - e);
        b = a;
        e = d;
      }
      if (b + k != trimx) {
        if (P.trace_off + atlen - 2 < 0) {
          W.err |= ALN_ERR_POINTS;
          return 1;
        }
        atrace[--atlen] = (uint16_t)(b - trimy);
        atrace[--atlen] = (uint16_t)(trimd - e);
      } else if (b != trimy) {
        atrace[atlen + 1] = (uint16_t)(atrace[atlen + 1] + (b - trimy));
        atrace[atlen] = (uint16_t)(atrace[atlen] + (trimd - e));
      }
    }
    P.abpos = trimx;
    P.bbpos = trimy;
    P.diffs = P.diffs + trimd;
    P.tlen = P.tlen - atlen;
    P.trace_off = P.trace_off + atlen;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Local_Alignment (lib/align.c:1423-1576).  `acomp` = ACOMP_FLAG: A is the
// complemented contig; the result is reported in forward A coordinates with
// the trace reversed.  P.trace_off is set here (maxtp into the points arena).
// ---------------------------------------------------------------------------
PGA_HD int local_alignment(WaveWork &W, const AlignSpec &spec, const Seq &A, const Seq &B, bool acomp,
                           Path &P, int low, int hgh, int anti, int lbord, int hbord) {
  int aoff, minp, maxp;
  bool fshort, rshort;
  int maxtp = 2 * (A.len / spec.trace_space + 2);
  if (2 * (int64_t)maxtp > W.point_cap) {
    W.err |= ALN_ERR_POINTS;
    return 1;
  }
  P.trace_off = maxtp;
  const bool selfie = false;  // aseq and bseq are always distinct buffers here
  while (((anti - hgh) >> 1) < 0) hgh -= 1;
  if (lbord < 0)
    minp = (selfie && low >= 0) ? 1 : -I32MAX;
  else
    minp = low - lbord;
  if (hbord < 0)
    maxp = (selfie && hgh <= 0) ? -1 : I32MAX;
  else
    maxp = hgh + hbord;
  aoff = acomp ? A.len % spec.trace_space : 0;

  if (forward_wave(W, spec, A, B, P, &low, hgh, anti, minp, maxp, aoff)) return 1;
  fshort = ((P.aepos + P.bepos) - anti < DUB_TRIM);
  if (reverse_wave(W, spec, A, B, P, low, low, anti, minp, maxp, aoff)) return 1;
  rshort = (anti - (P.abpos + P.bbpos) < DUB_TRIM);
  if (fshort) {
    if (rshort) {
      P.aepos = P.abpos = (P.abpos + P.aepos) >> 1;
      P.bepos = P.bbpos = (P.bbpos + P.bepos) >> 1;
      P.tlen = 0;
    } else {
      low = P.abpos - P.bbpos;
      anti = P.abpos + P.bbpos;
      P.tlen = 0;  // the trace keeps the start the reverse half left (lib/align.c:1509-1516)
      if (forward_wave(W, spec, A, B, P, &low, low, anti, minp, maxp, aoff)) return 1;
    }
  } else if (rshort) {
    low = P.aepos - P.bepos;
    anti = P.aepos + P.bepos;
    P.tlen = 0;
    P.diffs = 0;
    if (reverse_wave(W, spec, A, B, P, low, low, anti, minp, maxp, aoff)) return 1;
  }
  if (acomp) {
    uint16_t *trace = W.points + P.trace_off;
    int i = P.abpos;
    P.abpos = A.len - P.aepos;
    P.aepos = A.len - i;
    i = P.bbpos;
    P.bbpos = B.len - P.bepos;
    P.bepos = B.len - i;
    i = P.tlen - 2;
    int j = 0;
    while (j < i) {
      uint16_t p = trace[i];
      trace[i] = trace[j];
      trace[j] = p;
      p = trace[i + 1];
      trace[i + 1] = trace[j + 1];
      trace[j + 1] = p;
      i -= 2;
      j += 2;
    }
  }
  return 0;
}


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
  int *tmp;  // ovl_cap ints for the merge sort in finish_pair (nullptr: insertion sort)
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

// entwine (src/fastga_pipeline.c:505-570): whether two alignments' trace
// points cross; returns the signed minimal b-distance, *where the a position
// of a crossing (or -1).
PGA_HD int entwine(const Ovl &J, const uint8_t *jtrace, const Ovl &K, const uint8_t *ktrace, int *where) {
  int ac, b2, y2, yp, ae, i, j, k, mn;
  *where = -1;
  y2 = J.bbpos;
  b2 = K.bbpos;
  j = J.abpos / TSPACE;
  k = K.abpos / TSPACE;
  ac = k * TSPACE;
  j = 1 + 2 * (k - j);
  k = 1;
  for (i = 1; i < j; i += 2) y2 += jtrace[i];
  if (j == 1)
    yp = y2 + (jtrace[j] * (K.abpos - J.abpos)) / (ac + TSPACE - J.abpos);
  else
    yp = y2 + (jtrace[j] * (K.abpos - ac)) / TSPACE;
  mn = b2 - yp;
  ae = J.aepos;
  if (ae > K.aepos) ae = K.aepos;
  for (ac += TSPACE; ac < ae; ac += TSPACE) {
    y2 += jtrace[j];
    b2 += ktrace[k];
    j += 2;
    k += 2;
    i = b2 - y2;
    if (mn < 0 && mn < i) {
      if (i >= 0) mn = 0; else mn = i;
    } else if (mn > 0 && mn > i) {
      if (i <= 0) mn = 0; else mn = i;
    }
    if (i == 0) *where = ac;
  }
  ac -= TSPACE;
  if (ae == J.aepos) {
    y2 = J.bepos;
    if (K.aepos >= ac)
      b2 += (ktrace[k] * (ae - ac)) / TSPACE;
    else
      b2 += (ktrace[k] * (ae - ac)) / (K.aepos - ac);
  } else {
    b2 = K.bepos;
    if (J.aepos >= ac)
      y2 += (jtrace[j] * (ae - ac)) / TSPACE;
    else
      y2 += (jtrace[j] * (ae - ac)) / (J.aepos - ac);
  }
  i = b2 - y2;
  if (mn < 0 && mn < i) {
    if (i >= 0) mn = 0; else mn = i;
  } else if (mn > 0 && mn > i) {
    if (i <= 0) mn = 0; else mn = i;
  }
  return mn;
}

// Sort, duplicate/containment elimination, entwine merging and box
// elimination of a pair's candidates (src/fastga_pipeline.c:815-980).  On
// return perm[0..nov) lists the candidates by abpos (stable) and survivors
// are those without ELIMINATED.
PGA_HD void finish_pair(OvlArena &O) {
  const int64_t nlas = O.nov;
  Ovl *ov = O.ovl;
  int *perm = O.perm;
  for (int64_t j = 0; j < nlas; j++) perm[j] = (int)j;
  // stable sort by abpos (ALIGN_SORT under glibc's stable qsort): bottom-up
  // merge sort through O.tmp, or insertion sort without it
  if (O.tmp != nullptr && nlas > 16) {
    int *src = perm, *dst = O.tmp;
    for (int64_t w = 1; w < nlas; w <<= 1) {
      for (int64_t lo = 0; lo < nlas; lo += 2 * w) {
        int64_t mid = lo + w < nlas ? lo + w : nlas;
        int64_t hi = lo + 2 * w < nlas ? lo + 2 * w : nlas;
        int64_t i = lo, j = mid, k = lo;
        while (i < mid && j < hi) dst[k++] = (ov[src[j]].abpos < ov[src[i]].abpos) ? src[j++] : src[i++];
        while (i < mid) dst[k++] = src[i++];
        while (j < hi) dst[k++] = src[j++];
      }
      int *x = src;
      src = dst;
      dst = x;
    }
    if (src != perm)
      for (int64_t j = 0; j < nlas; j++) perm[j] = src[j];
  } else {
    for (int64_t j = 1; j < nlas; j++) {
      int x = perm[j];
      int64_t k = j - 1;
      while (k >= 0 && ov[perm[k]].abpos > ov[x].abpos) {
        perm[k + 1] = perm[k];
        k--;
      }
      perm[k + 1] = x;
    }
  }
  for (int64_t j = nlas - 1; j >= 0; j--) {
    Ovl &o = ov[perm[j]];
    for (int64_t k = j + 1; k < nlas; k++) {
      Ovl &w = ov[perm[k]];
      if (o.aepos <= w.abpos) break;
      if (w.flags & ELIMINATED) continue;
      if (o.abpos == w.abpos && o.bbpos == w.bbpos) {
        if (o.aepos == w.aepos && o.bepos == w.bepos) {
          if (o.diffs < w.aepos) {
            w.flags |= ELIMINATED;
            continue;
          } else {
            o.flags |= ELIMINATED;
            break;
          }
        } else {
          if (o.aepos > w.aepos) {
            w.flags |= ELIMINATED;
            continue;
          } else {
            o.flags |= ELIMINATED;
            break;
          }
        }
      } else if (o.aepos == w.aepos && o.bepos == w.bepos) {
        if (o.abpos < w.abpos) {
          w.flags |= ELIMINATED;
          continue;
        } else {
          o.flags |= ELIMINATED;
          break;
        }
      }
    }
  }
  for (int64_t j = nlas - 1; j >= 0; j--) {
    Ovl &o = ov[perm[j]];
    if (o.flags & ELIMINATED) continue;
    for (int64_t k = j + 1; k < nlas; k++) {
      Ovl &w = ov[perm[k]];
      int where, dist;
      if (o.aepos <= w.abpos) break;
      if (w.flags & ELIMINATED) continue;
      if (o.bepos <= w.bbpos || o.bbpos >= w.bepos) continue;
      const uint8_t *otrace = O.bytes + o.toff;
      const uint8_t *wtrace = O.bytes + w.toff;
      dist = entwine(o, otrace, w, wtrace, &where);
      if (where != -1) {
        int ocut = 2 * (((where - o.abpos) - 1) / TSPACE + 1);
        int wcut = 2 * (((where - w.abpos) - 1) / TSPACE + 1);
        int ntlen = ocut + (w.tlen - wcut);
        if (!O.reserve(ntlen, false)) {
          O.err |= ALN_ERR_TRACE;
          return;
        }
        uint8_t *nt = O.bytes + O.nbyte;
        int d = 0, h = 0;
        for (int g = 0; g < ocut; g += 2) {
          d += (nt[h] = otrace[g]);
          nt[h + 1] = otrace[g + 1];
          h += 2;
        }
        for (int g = wcut; g < w.tlen; g += 2) {
          d += (nt[h] = wtrace[g]);
          nt[h + 1] = wtrace[g + 1];
          h += 2;
        }
        o.toff = O.nbyte;
        O.nbyte += ntlen;
        o.tlen = ntlen;
        o.diffs = d;
        o.aepos = w.aepos;
        o.bepos = w.bepos;
        w.flags |= ELIMINATED;
        continue;
      }
      if (dist != 0) {  // BOX_ELIM
        if ((o.aepos - o.abpos) + BOX_FUZZ >= w.aepos - w.abpos) {
          if (w.aepos <= o.aepos + BOX_FUZZ && w.bbpos >= o.bbpos - BOX_FUZZ && w.bepos <= o.bepos + BOX_FUZZ) {
            w.flags |= ELIMINATED;
            continue;
          }
        } else {
          if (o.aepos <= w.aepos + BOX_FUZZ && o.bbpos >= w.bbpos - BOX_FUZZ && o.bepos <= w.bepos + BOX_FUZZ &&
              o.abpos >= w.abpos - BOX_FUZZ) {
            o.flags |= ELIMINATED;
            continue;
          }
        }
      }
    }
  }
}

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

// The scalar aligner: Local_Alignment on one thread.
struct ScalarAligner {
  WaveWork &W;
  const AlignSpec &spec;
  PGA_HD int call(const Seq &A, const Seq &B, bool acomp, Path &P, int low, int hgh, int anti, int lbord,
                  int hbord) {
    return local_alignment(W, spec, A, B, acomp, P, low, hgh, anti, lbord, hbord);
  }
  PGA_HD const uint16_t *points() const { return W.points; }
  PGA_HD int err() const { return W.err; }
};

// align_contigs (src/fastga_pipeline.c:576-813) for one pair, leaving the
// candidates in O (finish_pair does the rest).  A is the anchor contig,
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

#undef PGA_VI

}  // namespace aln
}  // namespace pga
