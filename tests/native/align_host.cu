// Test-only host build of the shared chain driver (align_core.cuh) and the
// finishing step (finish.cuh, its lanes run one after another): runs the
// alignment stage of one unit on the CPU from diagonal-sorted seed panels so
// the restated algorithm can be compared with the reference's .1aln on a
// machine without a GPU.  Local_Alignment is the oracle's scalar
// restatement (oracle/scalar_align.cuh); the oracle's finishing step can
// stand in for the product's (aht_set_finish) and the two are compared on
// random candidate sets (aht_finish_check).  Not part of the product library.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "../../distributedpanga_b200/csrc/align_core.cuh"
#include "../../distributedpanga_b200/csrc/align_spec.h"
#include "../../distributedpanga_b200/csrc/finish.cuh"
#include "../../oracle/scalar_align.cuh"

using namespace pga::aln;
using pga::aln::oracle::ScalarAligner;
using pga::aln::oracle::WaveWork;

static int g_oracle_finish = 0;

static void finish(OvlArena &O) {
  if (g_oracle_finish) oracle::finish_pair(O);
  else finish_candidates(Lanes{}, O);
}

extern "C" {

// Which finishing step aht_align_unit uses: 0 the product's, 1 the oracle's.
void aht_set_finish(int use_oracle) { g_oracle_finish = use_oracle; }

// The finishing step of one candidate set, by the product's code (which = 0)
// or the oracle's (which = 1): n candidates rows6 (abpos aepos bbpos bepos
// diffs tlen) with trace bytes at toff in trace.  Writes the survivors in
// order (rows6 and their trace bytes, concatenated); returns 0, or 1 when
// the arena overflowed.
int aht_finish_check(int64_t n, const int32_t *rows6, const int64_t *toff, const uint8_t *trace, int64_t nbytes,
                     int which, int32_t *out_rows, int64_t *out_n, uint8_t *out_trace, int64_t *out_nbytes) {
  std::vector<Ovl> ov(n > 0 ? n : 1);
  std::vector<int> perm(n > 0 ? n : 1), tmp(n > 0 ? n : 1);
  const int64_t cap = 4 * nbytes + 4096;
  std::vector<uint8_t> bytes(cap);
  memcpy(bytes.data(), trace, nbytes);
  for (int64_t i = 0; i < n; i++) {
    const int32_t *r = rows6 + 6 * i;
    ov[i].abpos = r[0]; ov[i].aepos = r[1]; ov[i].bbpos = r[2]; ov[i].bepos = r[3];
    ov[i].diffs = r[4]; ov[i].tlen = r[5]; ov[i].toff = toff[i]; ov[i].flags = 0;
  }
  OvlArena O;
  O.ovl = ov.data(); O.perm = perm.data(); O.tmp = tmp.data(); O.ovl_cap = n;
  O.bytes = bytes.data(); O.byte_cap = cap; O.nbyte = nbytes; O.nov = n; O.err = 0;
  O.pool_next = nullptr; O.pool_cap = 0;
  if (which) oracle::finish_pair(O);
  else finish_candidates(Lanes{}, O);
  if (O.err) return 1;
  int64_t k = 0, b = 0;
  for (int64_t q = 0; q < n; q++) {
    const Ovl &o = ov[perm[q]];
    if (o.flags & ELIMINATED) continue;
    int32_t *r = out_rows + 6 * k;
    r[0] = o.abpos; r[1] = o.aepos; r[2] = o.bbpos; r[3] = o.bepos; r[4] = o.diffs; r[5] = o.tlen;
    memcpy(out_trace + b, bytes.data() + o.toff, o.tlen);
    b += o.tlen;
    k++;
  }
  *out_n = k;
  *out_nbytes = b;
  return 0;
}

// Decodes swide records of one unit (sorted panels) and aligns every
// (anchor, partner) pair in panel order.  Self pairs (comp == 0 and
// anchor == partner) start from self_entry[anchor] (its bepos on entry).
// Output: one row per surviving alignment, pair by pair, in each pair's
// output order: aread bread comp abpos aepos bbpos bepos diffs tlen
// followed by the trace bytes in `tr`.  Also per pair: anchor, partner,
// calls, exit bepos (pairs_out, 4 ints per pair).
//
// split > 0 runs every pair of two different contigs the way the GPU runs a
// large one: as consecutive seed ranges of `split` seeds, each moved forward
// to the next band start, aligned separately and their candidates
// concatenated in range order before the pair's sort / elimination step; the
// pair's exit bepos is the last range's with a call.
int aht_align_unit(const uint8_t *bps, int ncontig, const int64_t *clen, const int64_t *boff, const float *freq,
                   const uint8_t *rec, const int64_t *panel_off, int swide, int dbyte, int ctgb, int comp,
                   const int *self_entry, int vcap, int64_t cell_cap, int64_t ovl_cap,
                   int *rows, int64_t row_cap, int64_t *nrows, uint8_t *tr, int64_t tr_cap, int64_t *ntr,
                   int *pairs_out, int64_t pair_cap, int64_t *npairs, int64_t split) {
  int64_t maxctg = 0;
  for (int i = 0; i < ncontig; i++) maxctg = clen[i] > maxctg ? clen[i] : maxctg;
  std::vector<int16_t> score(32768), table(32768);
  AlignSpec spec;
  spec.trace_space = 100;
  spec.reach = 0;
  spec.ave_path = build_align_spec(freq, score.data(), table.data());
  spec.score = score.data();
  spec.table = table.data();
  // NUMERIC contigs with sentinels; A complemented for the C unit
  std::vector<std::vector<uint8_t>> fwd(ncontig), rc(ncontig);
  for (int c = 0; c < ncontig; c++) {
    int64_t n = clen[c];
    fwd[c].assign(n + 2, 4);
    for (int64_t i = 0; i < n; i++) fwd[c][i + 1] = (bps[boff[c] + (i >> 2)] >> (2 * (i & 3))) & 3;
    rc[c].assign(n + 2, 4);
    for (int64_t i = 0; i < n; i++) rc[c][i + 1] = 3 - fwd[c][n - i];
  }
  WaveWork W;
  std::vector<int> V(vcap), M(vcap), HA(vcap), NA(vcap);
  std::vector<uint64_t> T(vcap);
  std::vector<Pebble> cells(cell_cap);
  int64_t pcap = 4 * (maxctg / 100 + 4);
  std::vector<uint16_t> points(pcap);
  W.V = V.data(); W.M = M.data(); W.HA = HA.data(); W.NA = NA.data(); W.T = T.data();
  W.vcap = vcap; W.cells = cells.data(); W.cell_cap = cell_cap; W.points = points.data(); W.point_cap = pcap;
  W.err = 0;
  OvlArena O;
  std::vector<Ovl> ovl(ovl_cap);
  std::vector<int> perm(ovl_cap), tmp(ovl_cap);
  int64_t bcap = 64 * (maxctg / 100 + 4) + (1 << 20);
  std::vector<uint8_t> bytes(bcap);
  O.ovl = ovl.data(); O.perm = perm.data(); O.tmp = tmp.data(); O.ovl_cap = ovl_cap; O.bytes = bytes.data();
  O.byte_cap = bcap;
  O.err = 0;
  O.pool_next = nullptr;
  O.pool_cap = 0;
  // one range's candidates when split > 0
  OvlArena G;
  std::vector<Ovl> govl(split > 0 ? ovl_cap : 1);
  std::vector<uint8_t> gbytes(split > 0 ? bcap : 1);
  G.ovl = govl.data(); G.perm = nullptr; G.tmp = nullptr; G.ovl_cap = split > 0 ? ovl_cap : 0;
  G.bytes = gbytes.data(); G.byte_cap = split > 0 ? bcap : 0;
  G.err = 0;
  G.pool_next = nullptr;
  G.pool_cap = 0;
  Path path;
  memset(&path, 0, sizeof(path));
  *nrows = 0; *ntr = 0; *npairs = 0;
  const int64_t mask = ((int64_t)1 << (8 * ctgb - 1)) - 1;
  for (int a = 0; a < ncontig; a++) {
    int64_t lo = panel_off[a], hi = panel_off[a + 1];
    int64_t i = lo;
    while (i < hi) {
      int64_t jc = 0;
      memcpy(&jc, rec + i * swide + 2 + 2 * dbyte, ctgb);
      jc &= mask;
      int64_t j = i;
      std::vector<int64_t> anti, band;
      std::vector<uint8_t> lcp, dlow;
      while (j < hi) {
        int64_t x = 0;
        memcpy(&x, rec + j * swide + 2 + 2 * dbyte, ctgb);
        if ((x & mask) != jc) break;
        int64_t an = 0, bd = 0;
        memcpy(&an, rec + j * swide + 2, dbyte);
        memcpy(&bd, rec + j * swide + 2 + dbyte, dbyte);
        anti.push_back(an);
        band.push_back(bd);
        lcp.push_back(rec[j * swide]);
        dlow.push_back(rec[j * swide + 1]);
        j++;
      }
      PairSeeds S{anti.data(), band.data(), lcp.data(), dlow.data(), (int64_t)anti.size()};
      bool self = (!comp && jc == a);
      if (self && self_entry) path.bepos = self_entry[a];
      const std::vector<uint8_t> &as = comp ? rc[a] : fwd[a];
      Seq A{as.data() + 1, (int)clen[a]};
      Seq B{fwd[jc].data() + 1, (int)clen[jc]};
      PairResult R;
      ScalarAligner AL{W, spec};
      if (split <= 0 || self) {
        if (align_pair(S, comp != 0, self, A, B, maxctg, 2 * maxctg, AL, path, O, R)) return 100 + (W.err | O.err);
      } else {
        const int64_t n = S.n;
        auto band_start = [&](int64_t x) {
          while (x < n && x > 0 && S.band(x) == S.band(x - 1)) x++;
          return x < n ? x : n;
        };
        O.nov = 0;
        O.nbyte = 0;
        R.calls = 0;
        R.exit_bepos = path.bepos;
        for (int64_t lo = 0; lo < n; lo += split) {
          int64_t blo = band_start(lo), bhi = band_start(lo + split < n ? lo + split : n);
          PairResult Rg;
          if (align_pair(S, comp != 0, false, A, B, maxctg, 2 * maxctg, AL, path, G, Rg, 0, 1, blo, bhi))
            return 100 + (W.err | G.err);
          if (O.nov + G.nov > O.ovl_cap || O.nbyte + G.nbyte > O.byte_cap) return 300;
          for (int64_t q = 0; q < G.nov; q++) {
            Ovl o = G.ovl[q];
            memcpy(O.bytes + O.nbyte, G.bytes + o.toff, o.tlen);
            o.toff = O.nbyte;
            O.nbyte += o.tlen;
            O.ovl[O.nov++] = o;
          }
          R.calls += Rg.calls;
          if (Rg.calls > 0) R.exit_bepos = Rg.exit_bepos;
        }
      }
      finish(O);
      if (O.err) return 200 + O.err;
      if (*npairs < pair_cap) {
        int *p = pairs_out + 4 * (*npairs);
        p[0] = a; p[1] = (int)jc; p[2] = R.calls; p[3] = R.exit_bepos;
      }
      (*npairs)++;
      for (int64_t q = 0; q < O.nov; q++) {
        const Ovl &o = O.ovl[O.perm[q]];
        if (o.flags & ELIMINATED) continue;
        if (*nrows < row_cap) {
          int *r = rows + 9 * (*nrows);
          r[0] = a; r[1] = (int)jc; r[2] = comp; r[3] = o.abpos; r[4] = o.aepos; r[5] = o.bbpos; r[6] = o.bepos;
          r[7] = o.diffs; r[8] = o.tlen;
          if (*ntr + o.tlen <= tr_cap) memcpy(tr + *ntr, O.bytes + o.toff, o.tlen);
        }
        (*nrows)++;
        *ntr += o.tlen;
      }
      i = j;
    }
  }
  return 0;
}
}
