// TEST INFRASTRUCTURE ONLY (oracle): a scalar, statement-by-statement
// restatement of FastGA's wave aligner and of align_contigs' finishing step,
// used by the host test harness (tests/native/align_host.cu) to run the
// chain driver on the CPU and to check the product's finishing step
// (distributedpanga_b200/csrc/finish.cuh) against the reference's rules.
// Nothing in the product includes this file.
//
// Restates:
//   forward_wave / reverse_wave / Local_Alignment   lib/align.c:352-1576
//   entwine                                         src/fastga_pipeline.c:505-570
//   sort, duplicate / containment elimination, entwine merge,
//     box elimination                               src/fastga_pipeline.c:815-980
//
// Differences of representation only: per-diagonal wave vectors live in ring
// buffers indexed by diagonal & (vcap - 1) instead of a re-centred window (the
// values are the same; a band wider than vcap - 2 diagonals sets ALN_ERR_VCAP),
// and trace-point pebbles and trace points live in caller-provided arenas.
#pragma once
#include "../distributedpanga_b200/csrc/align_core.cuh"

namespace pga {
namespace aln {
namespace oracle {

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


#undef PGA_VI

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


}  // namespace oracle
}  // namespace aln
}  // namespace pga
