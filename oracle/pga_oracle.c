/* CPU restatement of DistributedPanGA's alignment path up to the diagonal
 * sort.  TEST INFRASTRUCTURE ONLY -- see pga_oracle.h.  Every function cites
 * the reference lines it restates. */
#include "pga_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define KMER    40
#define KBYTES  10
#define TMER    12
#define SMER     8

/* The syncmer hash's 4-mer scramble table.  It is part of the definition of
 * the closed-syncmer selection (src/tables.c:5-22, the same table as FastGA's
 * GIXmake), so the values must be identical; nothing else is shared. */
static const uint8_t TMAP[256] = {
  0xff,0xd4,0xf5,0xfd,0xe4,0xad,0x21,0xa5,0xed,0x64,0xbf,0xa9,0xf3,0x70,0xd6,0xf0,
  0xca,0x89,0xcb,0xc9,0x82,0x9d,0x13,0x79,0x0a,0x0f,0x25,0x19,0x3e,0x47,0xa3,0xa8,
  0xf9,0x5e,0xe8,0xa1,0xb0,0x71,0x1d,0x8c,0xde,0x69,0xe7,0x7c,0x56,0x3f,0x90,0xa4,
  0xeb,0x45,0x59,0xf1,0x97,0x4c,0x08,0xa0,0xb8,0x4a,0x86,0xc8,0xcd,0x98,0x7d,0xfc,
  0xef,0x4d,0x83,0x7e,0xdc,0x66,0x2b,0x8e,0xe0,0xa7,0xd0,0xa2,0x88,0x5f,0x7f,0xd9,
  0x9b,0x78,0xd1,0x8b,0xc3,0x8f,0x2d,0xe6,0x18,0x27,0x2c,0x24,0x94,0xb7,0xce,0xbd,
  0x0d,0x04,0x1c,0x09,0x16,0x23,0x00,0x1e,0x1a,0x29,0x2e,0x15,0x01,0x10,0x2a,0x20,
  0xbe,0x31,0x43,0x58,0xc2,0xaa,0x1f,0xe5,0xc5,0x9e,0xcf,0xc6,0x68,0xb2,0x80,0xf4,
  0xf8,0x53,0xb6,0x93,0x76,0x37,0x11,0x40,0xda,0x51,0xba,0x46,0x42,0x30,0x60,0x6d,
  0x5c,0x39,0x9f,0x48,0x6c,0x62,0x28,0x67,0x06,0x12,0x26,0x0e,0x33,0x50,0xa6,0x63,
  0xdd,0x3b,0xab,0x4b,0x72,0x5b,0x22,0x6f,0xb4,0x61,0x92,0x99,0x36,0x38,0x65,0xac,
  0x4f,0x2f,0x32,0x44,0x54,0x3c,0x03,0x5d,0x73,0x3a,0x77,0x84,0x8d,0x4e,0x49,0xd2,
  0xfb,0x91,0x6a,0xcc,0x8a,0x35,0x02,0x55,0x7a,0x34,0x96,0x3d,0xd3,0x41,0x85,0xf2,
  0xb1,0x75,0xc4,0xb5,0xbb,0xb3,0x1b,0xd5,0x07,0x05,0x17,0x0b,0x7b,0xd7,0xdf,0xea,
  0xe3,0x57,0xc0,0x95,0x9c,0x6e,0x14,0xae,0xb9,0x6b,0xc1,0x81,0x87,0x74,0xd8,0xe2,
  0xec,0x52,0xbc,0xe9,0xe1,0xdb,0x0c,0xf7,0xaf,0x5a,0x9a,0xc7,0xfa,0xf6,0xee,0xfe };

const uint8_t *orc_tmap(void) { return TMAP; }

/* Reverse complement of a 4-mer packed MSB-first (first base in bits 7:6):
 * complement each base (3 - b) and reverse the order. */
static int rc4(int x)
{ int y = 0, i;
  for (i = 0; i < 4; i++)
    { y = (y << 2) | (3 - (x & 3));
      x >>= 2;
    }
  return y;
}

static int bytes_inclusive(int64_t maxv)
{ int b = 0;
  int64_t cum = 1;
  while (cum < maxv + 1) { cum *= 256; b += 1; }
  return b;
}

void orc_record_sizing(int ncontig, int64_t maxctg, int *posb, int *ctgb, int *rsize)
{ *posb  = bytes_inclusive(maxctg);                 /* src/record.c:29 */
  *ctgb  = bytes_inclusive(2 * (int64_t) ncontig - 1); /* src/record.c:35 */
  *rsize = 1 + KBYTES + 1 + *posb + *ctgb;          /* src/record.c:36 */
}

static inline int base_at(const uint8_t *bps, int64_t boff, int64_t i)
{ return (bps[boff + (i >> 2)] >> (2 * (i & 3))) & 3; }

static inline int quad(const uint8_t *s, int64_t i)   /* 4-mer at i, MSB-first */
{ return (s[i] << 6) | (s[i+1] << 4) | (s[i+2] << 2) | s[i+3]; }

/* Canonical hash of the 8-mer at i (src/extract.c:147-165; contract
 * tests/support/ref_syncmer.h:20-43): min of the forward hash
 * TMap[q(i)]<<8 | TMap[q(i+4)] and the reverse-complement hash
 * TMap[rc(q(i+4))]<<8 | TMap[rc(q(i))]. */
static inline int hash8(const uint8_t *s, int64_t i)
{ int a = quad(s, i), b = quad(s, i + 4);
  int f = (TMAP[a] << 8) | TMAP[b];
  int r = (TMAP[rc4(b)] << 8) | TMAP[rc4(a)];
  return f < r ? f : r;
}

static void emit(uint8_t *out, int64_t cap, int64_t k, int rsize, int posb, int ctgb,
                 int contig, int64_t pos, int strand, const uint8_t *kmer)
{ uint8_t *r;
  int64_t cs;
  int b;
  if (out == NULL || k >= cap) return;
  r = out + k * rsize;                              /* src/extract.c:294-323 */
  r[0] = 0;
  memcpy(r + 1, kmer, KBYTES);
  r[11] = 0;
  for (b = 0; b < posb; b++) r[12 + b] = (uint8_t) (pos >> (8 * b));
  cs = contig;
  if (strand) cs |= ((int64_t) 1) << (8 * ctgb - 1);
  for (b = 0; b < ctgb; b++) r[12 + posb + b] = (uint8_t) (cs >> (8 * b));
}

int64_t orc_extract(const uint8_t *bps, int ncontig, const int64_t *clen, const int64_t *boff,
                    int posb, int ctgb, uint8_t *out, int64_t cap)
{ int rsize = 1 + KBYTES + 1 + posb + ctgb;
  int64_t k = 0;
  int c;
  uint8_t *s = NULL;
  int64_t smax = 0;

  for (c = 0; c < ncontig; c++)
    { int64_t len = clen[c], i, j;
      if (boff[c] < 0 || len < TMER) continue;      /* src/extract.c:101 */
      if (len > smax)
        { free(s);
          smax = len;
          s = malloc((size_t) smax + 8);
        }
      for (i = 0; i < len; i++) s[i] = (uint8_t) base_at(bps, boff[c], i);
      for (j = 0; j <= len - TMER; j++)
        { int h[5], t, m, sel;
          uint8_t km[KBYTES];
          for (t = 0; t < 5; t++) h[t] = hash8(s, j + t);
          m = h[0];
          for (t = 1; t < 5; t++) if (h[t] < m) m = h[t];
          /* closed syncmer: the earliest minimum is the first 8-mer, or the
             last 8-mer ties the minimum (tests/CATALOG.md:140-150) */
          sel = (h[0] == m) || (h[4] == m);
          if (!sel) continue;
          if (j <= len - KMER)                      /* forward 40-mer at j, src/pack.c:29-42 */
            { for (t = 0; t < KBYTES; t++) km[t] = (uint8_t) quad(s, j + 4 * t);
              emit(out, cap, k++, rsize, posb, ctgb, c, j, 0, km);
            }
          if (j >= KMER - TMER)                     /* RC of [j-28, j+12) stored at j+12, src/pack.c:64-78 */
            { for (t = 0; t < KBYTES; t++) km[t] = (uint8_t) rc4(quad(s, j - 28 + 36 - 4 * t));
              emit(out, cap, k++, rsize, posb, ctgb, c, j + TMER, 1, km);
            }
        }
    }
  free(s);
  return k;
}

/* ---- sort + LCP ---------------------------------------------------------- */

static int Sort_Rsize;

static int rec_cmp(const void *x, const void *y)
{ const uint8_t *a = x, *b = y;
  int c = memcmp(a + 1, b + 1, KBYTES), i;
  if (c) return c;
  for (i = Sort_Rsize - 1; i >= 12; i--)             /* payload as one LE integer */
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  return 0;
}

int orc_lcp_bases(const uint8_t *a, const uint8_t *b)
{ int i, k;
  for (i = 0; i < KBYTES; i++)                       /* src/sort.c:16-32 */
    if (a[i] != b[i])
      { int d = a[i] ^ b[i];
        for (k = 0; k < 4; k++)
          if ((d >> (6 - 2 * k)) & 3) return 4 * i + k;
      }
  return KMER;
}

void orc_sort_records(uint8_t *rec, int64_t n, int rsize)
{ int64_t i;
  Sort_Rsize = rsize;
  qsort(rec, (size_t) n, (size_t) rsize, rec_cmp);
  if (n == 0) return;
  rec[0] = 0;                                        /* src/sort.c:38-57 */
  for (i = 1; i < n; i++)
    rec[i * rsize] = (uint8_t) orc_lcp_bases(rec + (i - 1) * rsize + 1, rec + i * rsize + 1);
}

/* ---- k-mer table view ---------------------------------------------------- */

int64_t orc_build_adapter(const uint8_t *rec, int64_t n, int rsize, int posb, int ctgb,
                          uint8_t *entries, int64_t *cum)
{ int ebytes = 7 + 1 + 1 + posb + ctgb;             /* src/kmer_adapter.c:17-18 */
  int64_t i, run = 0, best = 0, acc;
  int prev = -1;

  memset(cum, 0, sizeof(int64_t) << 24);
  for (i = 0; i < n; i++)
    { const uint8_t *s = rec + i * rsize;
      uint8_t *d = entries + i * ebytes;
      int p = (s[1] << 16) | (s[2] << 8) | s[3];
      if (p == prev) run += 1;
      else { if (run > best) best = run; run = 1; prev = p; }
      memcpy(d, s + 4, 7);                           /* src/kmer_adapter.c:60-65 */
      d[7] = 0;
      d[8] = s[0];
      memcpy(d + 9, s + 12, (size_t) (posb + ctgb));
      cum[p] += 1;
    }
  if (run > best) best = run;
  acc = 0;
  for (i = 0; i < (1 << 24); i++) { acc += cum[i]; cum[i] = acc; }   /* src/kmer_adapter.c:71-86 */
  return best;
}

/* ---- adaptamer merge ----------------------------------------------------- */

static int put_seed(uint8_t *buf, int64_t cap, int64_t *len, int sbytes, int plen,
                    const uint8_t *apay, const uint8_t *bpay, int pay)
{ if (*len + sbytes <= cap && buf != NULL)
    { uint8_t *d = buf + *len;
      d[0] = (uint8_t) plen;
      memcpy(d + 1, apay, (size_t) pay);
      memcpy(d + 1 + pay, bpay, (size_t) pay);
    }
  *len += sbytes;
  return 0;
}

int orc_merge(const uint8_t *entries, const int64_t *cum, int64_t n, int ebytes, int posb, int ctgb,
              int freq, int ncontig,
              uint8_t *nseed, int64_t ncap, int64_t *nlen,
              uint8_t *cseed, int64_t ccap, int64_t *clen_out,
              int64_t *nbuck, int64_t *cbuck)
{ const int LCPO = 8, PAYO = 9;                      /* entry offsets, src/pga-mpi-merge.c:71-90 */
  int pay = posb + ctgb;
  int sbytes = 1 + 2 * pay;
  int sgn = pay - 1;                                 /* payload byte holding the strand bit */
  int64_t g0 = 0;
  int p;
  uint8_t *cache;
  int64_t gmax = 0;

  (void) n;
  *nlen = 0;
  *clen_out = 0;
  memset(nbuck, 0, sizeof(int64_t) * (size_t) ncontig);
  memset(cbuck, 0, sizeof(int64_t) * (size_t) ncontig);

  /* largest prefix group sizes the cache (src/fastga_pipeline.c:469-472) */
  for (p = 0; p < (1 << 24); p++)
    { int64_t e = cum[p] - (p ? cum[p - 1] : 0);
      if (e > gmax) gmax = e;
    }
  cache = malloc((size_t) (gmax + 1) * (size_t) ebytes);

  /* Walk every non-empty 24-bit prefix group in order, restating
     new_self_merge_thread (src/fastga_pipeline.c:245-412) for NTHREADS = 1. */
  for (p = 0; p < (1 << 24); p++)
    { int64_t gn = cum[p] - g0, i;
      int64_t vlcp[KMER + 2];
      int64_t rcur, rend;
      int plen, eorun;
      if (gn <= 0) continue;
      memcpy(cache, entries + g0 * ebytes, (size_t) (gn * ebytes));
      g0 = cum[p];
      cache[gn * ebytes + LCPO] = 11;               /* end-of-group marker, :301 */
#define LCP(k) (cache[(k) * ebytes + LCPO])
      /* group start, :303-308 */
      rcur = 0;
      rend = 1;
      plen = LCP(rend);
      for (i = LCP(rcur); i <= plen; i++) vlcp[i] = rcur;
      eorun = (plen <= 11);
      for (i = 0; i < gn; i++)
        { int64_t low, hgh, top;
          if (i > 0)                                 /* :310-327 */
            { if (eorun) plen = LCP(i);
              rend += 1;
              if (LCP(rend) < plen) eorun = 1;
              else if (LCP(rend) == plen) eorun = 0;
              else
                { int q;
                  rcur = rend - 1;
                  for (q = plen + 1; q <= LCP(rend); q++) vlcp[q] = rcur;
                  eorun = 0;
                  plen = LCP(rend);
                }
            }
          low = vlcp[plen];                          /* :329-340 */
          hgh = rend;
          top = low + freq;
          if (!eorun)
            { do
                { hgh += 1;
                  if (hgh > top) break;
                }
              while (LCP(hgh) >= plen);
            }
          if (hgh >= top) continue;
          { uint8_t a[8], *b;                        /* :343-403 */
            int64_t q, icont = 0;
            int isign;
            memcpy(a, cache + i * ebytes + PAYO, (size_t) pay);
            isign = a[sgn] & 0x80;
            a[sgn] &= 0x7f;
            memcpy(&icont, a + posb, (size_t) ctgb);
            for (q = low; q < hgh; q++)
              { int jsign;
                if (q == i) continue;
                b = cache + q * ebytes + PAYO;
                jsign = b[sgn] & 0x80;
                if (isign == jsign)
                  { put_seed(nseed, ncap, nlen, sbytes, plen, a, b, pay); nbuck[icont] += 1; }
                else
                  { put_seed(cseed, ccap, clen_out, sbytes, plen, a, b, pay); cbuck[icont] += 1; }
              }
          }
        }
#undef LCP
    }
  free(cache);
  return (*nlen > ncap || *clen_out > ccap) ? -1 : 0;
}

/* ---- reimport + diagonal sort ------------------------------------------- */

void orc_diag_sizing(int64_t maxctg, int ctgb, int *dbyte, int *swide)
{ int64_t maxdag = 2 * maxctg, cum = 1;             /* src/pga-mpi-merge.c:415-425 */
  int d = 0;
  while (cum < maxdag) { cum *= 256; d += 1; }
  *dbyte = d;
  *swide = 2 * d + ctgb + 2;                         /* src/fastga_pipeline.c:1736 */
}

static int Diag_Swide;

static int diag_cmp(const void *x, const void *y)    /* lib/RSDsort.c: key read backwards */
{ const uint8_t *a = x, *b = y;
  int i;
  for (i = Diag_Swide - 1; i >= 0; i--)
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  return 0;
}

int orc_reimport_sort(const uint8_t *seeds, int64_t len, int posb, int ctgb, int comp,
                      int ncontig, int64_t amxpos, int dbyte,
                      uint8_t *out, int64_t *panel_off)
{ int pay = posb + ctgb, sbytes = 1 + 2 * pay;
  int swide = 2 * dbyte + ctgb + 2;
  int64_t ns = len / sbytes, s, *fill;
  int64_t bmxpos = amxpos, maxdag = amxpos + bmxpos;
  int64_t jmask = (((int64_t) 1) << (8 * ctgb - 1)) - 1;
  int c;

  memset(panel_off, 0, sizeof(int64_t) * (size_t) (ncontig + 1));
  for (s = 0; s < ns; s++)
    { int64_t icont = 0;
      memcpy(&icont, seeds + s * sbytes + 1 + posb, (size_t) ctgb);
      panel_off[icont + 1] += 1;
    }
  for (c = 0; c < ncontig; c++) panel_off[c + 1] += panel_off[c];
  fill = malloc(sizeof(int64_t) * (size_t) (ncontig + 1));
  memcpy(fill, panel_off, sizeof(int64_t) * (size_t) (ncontig + 1));

  for (s = 0; s < ns; s++)                           /* src/fastga_pipeline.c:1418-1447 */
    { const uint8_t *b = seeds + s * sbytes;
      int64_t ipost = 0, icont = 0, jpost = 0, jcont = 0, diag, anti, band;
      uint8_t *x;
      memcpy(&ipost, b + 1, (size_t) posb);
      memcpy(&icont, b + 1 + posb, (size_t) ctgb);
      memcpy(&jpost, b + 1 + pay, (size_t) posb);
      memcpy(&jcont, b + 1 + pay + posb, (size_t) ctgb);
      jcont &= jmask;
      x = out + swide * fill[icont]++;
      x[0] = b[0];
      if (comp) { diag = maxdag - (ipost + jpost); anti = amxpos - (ipost - jpost); }
      else      { diag = bmxpos + (ipost - jpost); anti = ipost + jpost; }
      band = diag >> 6;
      x[1] = (uint8_t) (diag - (band << 6));
      memcpy(x + 2, &anti, (size_t) dbyte);
      memcpy(x + 2 + dbyte, &band, (size_t) dbyte);
      memcpy(x + 2 + 2 * dbyte, &jcont, (size_t) ctgb);
    }
  free(fill);

  Diag_Swide = swide;
  for (c = 0; c < ncontig; c++)
    { int64_t a = panel_off[c], e = panel_off[c + 1];
      if (e - a > 1) qsort(out + a * swide, (size_t) (e - a), (size_t) swide, diag_cmp);
    }
  return swide;
}

/* ---- Create_GDB's FASTA reader ------------------------------------------ */

/* Base value of a sequence character (lib/GDB.c:350-367): A/a 0, C/c 1,
 * G/g 2, T/t 3, N/n 4 (not a base), every other character 0. */
static int fa_value(int c)
{ switch (c)
    { case 'C': case 'c': return 1;
      case 'G': case 'g': return 2;
      case 'T': case 't': return 3;
      case 'N': case 'n': return 4;
      default:            return 0;
    }
}

static int fa_isspace(int c)
{ return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

typedef struct
  { int64_t *ctg4, ctg_cap, ncontig;
    uint8_t *bps;
    int64_t  bps_cap, boff;     /* bytes written so far */
    int      m;                 /* bits used in the partial byte */
    uint8_t  byte;
    int64_t  count[4];
    int64_t  maxctg;
    int      over;
  } FaState;

/* Appends base v to the current contig's bytes (lib/GDB.c:960-977). */
static void fa_put(FaState *F, int v)
{ F->byte |= (uint8_t) (v << F->m);
  if (F->m == 6)
    { if (F->boff < F->bps_cap) F->bps[F->boff] = F->byte; else F->over = 1;
      F->boff += 1;
      F->m = 0;
      F->byte = 0;
    }
  else
    F->m += 2;
  F->count[v] += 1;
}

/* Ends the current contig: flushes its partial byte and records it
 * (lib/GDB.c:897-956). */
static void fa_close(FaState *F, int64_t clen, int64_t sbeg, int64_t bpos, int64_t scaf)
{ if (F->m > 0)
    { if (F->boff < F->bps_cap) F->bps[F->boff] = F->byte; else F->over = 1;
      F->boff += 1;
    }
  F->byte = 0;
  F->m = 0;
  if (F->ncontig < F->ctg_cap)
    { int64_t *c = F->ctg4 + 4 * F->ncontig;
      c[0] = clen;
      c[1] = bpos;
      c[2] = sbeg;
      c[3] = scaf;
    }
  else
    F->over = 1;
  F->ncontig += 1;
  if (clen > F->maxctg) F->maxctg = clen;
}

/* The reader works line by line as read_line (lib/GDB.c:372-439) does: a line
 * must end with a new-line.  Within a scaffold the N runs of its lines join
 * into one run across line ends (lib/GDB.c:850-876): a run of length L that
 * is followed by a base is a gap, filled with L A's when L < nthr
 * (lib/GDB.c:879-897) and otherwise ending the current contig
 * (lib/GDB.c:898-956), so a scaffold that opens with such a run has an
 * empty first contig; the run that ends a scaffold is dropped
 * (lib/GDB.c:853-857, lib/GDB.c:870-874, lib/GDB.c:947-950).  A scaffold
 * without any base is an error (lib/GDB.c:1039-1043).  NUL and non-ASCII
 * bytes, which the reference does not read as characters, are refused. */
int orc_fasta_gdb(const char *text, int64_t n, int nthr,
                  int64_t *scf4, int64_t scf_cap, int64_t *ctg4, int64_t ctg_cap,
                  char *hdr, int64_t hdr_cap, uint8_t *bps, int64_t bps_cap,
                  int64_t *sizes6, int64_t *count4, char *err, int errlen)
{ FaState F;
  int64_t pos, nscaff, hdrtot, i;
  int     over;

  memset(&F, 0, sizeof(F));
  F.ctg4 = ctg4;
  F.ctg_cap = ctg_cap;
  F.bps = bps;
  F.bps_cap = bps_cap;
  nscaff = 0;
  hdrtot = 0;
  over = 0;
  if (err && errlen > 0) err[0] = '\0';

  if (n <= 0)
    { if (err) snprintf(err, errlen, "input is empty");
      return -1;
    }
  for (i = 0; i < n; i++)
    if (text[i] == 0 || (uint8_t) text[i] >= 128)
      { if (err) snprintf(err, errlen, "byte %lld is NUL or not ASCII", (long long) i);
        return -1;
      }
  if (text[n - 1] != '\n')
    { if (err) snprintf(err, errlen, "last line does not end with new-line");
      return -1;
    }
  if (text[0] != '>')
    { if (err) snprintf(err, errlen, "first header is missing");
      return -1;
    }

  pos = 0;
  while (pos < n)
    { /* header line: text after '>' and any white space (lib/GDB.c:815-834) */
      int64_t e = pos;
      int64_t s, len, clen, spos, bpos, pend;
      while (text[e] != '\n') e += 1;
      len = e - pos;
      for (s = 1; s < len; s++)
        if (!fa_isspace(text[pos + s])) break;
      if (nscaff < scf_cap)
        { scf4[4 * nscaff + 0] = F.ncontig;
          scf4[4 * nscaff + 3] = hdrtot;
        }
      else
        over = 1;
      if (hdrtot + (len - s) + 1 <= hdr_cap)
        { memcpy(hdr + hdrtot, text + pos + s, (size_t) (len - s));
          hdr[hdrtot + len - s] = '\0';
        }
      else
        over = 1;
      hdrtot += len - s + 1;
      pos = e + 1;

      /* sequence lines up to the next header or the end */
      clen = 0;
      spos = 0;
      bpos = F.boff;
      pend = 0;
      while (pos < n && text[pos] != '>')
        { for (; text[pos] != '\n'; pos++)
            { int v = fa_value(text[pos]);
              if (v == 4)
                { pend += 1;
                  continue;
                }
              if (pend > 0)
                { if (pend < nthr)
                    { int64_t x;
                      for (x = 0; x < pend; x++) fa_put(&F, 0);
                      clen += pend;
                    }
                  else
                    { fa_close(&F, clen, spos, bpos, nscaff);
                      spos += clen + pend;
                      bpos = F.boff;
                      clen = 0;
                    }
                  pend = 0;
                }
              fa_put(&F, v);
              clen += 1;
            }
          pos += 1;
        }
      fa_close(&F, clen, spos, bpos, nscaff);
      spos += clen;
      if (spos == 0)
        { if (err) snprintf(err, errlen, "scaffold %lld has no sequence", (long long) nscaff);
          return -1;
        }
      if (nscaff < scf_cap)
        { scf4[4 * nscaff + 1] = F.ncontig;
          scf4[4 * nscaff + 2] = spos;
        }
      nscaff += 1;
    }

  sizes6[0] = nscaff;
  sizes6[1] = F.ncontig;
  sizes6[2] = F.boff;
  sizes6[3] = hdrtot;
  sizes6[4] = F.maxctg;
  sizes6[5] = F.count[0] + F.count[1] + F.count[2] + F.count[3];
  for (i = 0; i < 4; i++) count4[i] = F.count[i];
  return (over || F.over) ? -2 : 0;
}
