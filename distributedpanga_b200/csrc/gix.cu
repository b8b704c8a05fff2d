// The GIX k-mer index on disk, as FastGA's GIXmake leaves it
// (notes/GIXmake_annotated.c:1529-1615; read back by src/fastga_order_core.c:11-52
// and by FastGA):
//
//   <dir>/<root>.gix         int K, int NPARTS, int 1, int 3,
//                            int64 cumulative count per 24-bit prefix (2^24),
//                            int PostBytes, int ContBytes, int NPARTS,
//                            int64 largest prefix group, int 0 (frequency
//                            cutoff), int ncontig, int order[ncontig]
//                            (contigs longest first), int64 -1
//   <dir>/.<root>.ktab.<p>   int K, int64 entries, then the entries of part
//                            p (1-based) in sorted order
//
// An entry is k-mer bytes 3..9, the mask byte, the LCP byte and the payload
// (position, contig|strand, little-endian) -- the k-mer table view's entry,
// except that GIXmake numbers a contig by its place in the longest-first
// order (notes/GIXmake_annotated.c:2037-2047: InvP).  A part holds whole
// 10-bit panels (the first five bases); within a run of equal k-mers the first
// entry carries the LCP to the previous k-mer and the others 40
// (notes/GIXmake_annotated.c:1224-1290).  The first entry of a part carries
// what GIXmake's part-by-part sort leaves there (lib/MSDsort.c:485-500): 0
// when the part's first panel holds k-mers, else the bases its panel shares
// with that first panel.  Host code only.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/pga_b200.h"

namespace {

constexpr int GIX_KMER = 40;
constexpr int PANEL_SHIFT = 14;          // 24-bit prefix -> 10-bit panel
constexpr int NPANEL = 1 << 10;

bool put(FILE *f, const void *p, size_t n) { return fwrite(p, 1, n, f) == n; }

// Leading equal bases of two panels (10 bits, the first base in the top two).
int panel_lcp(int x, int n) {
  if ((x & 0x300) != (n & 0x300)) return 0;
  int v = (x ^ n) & 0xff, z = 0;
  while (z < 4 && !(v & (0xc0 >> (2 * z)))) z++;
  return 1 + z;
}

}  // namespace

extern "C" int pga_write_gix(const char *stem, int nparts, int post_bytes, int cont_bytes, int ncontig,
                             const int32_t *order, const int64_t *cum, int64_t largest, int64_t nentries,
                             const uint8_t *entries) {
  if (!stem || nparts < 1 || nparts > NPANEL || post_bytes < 1 || cont_bytes < 1 || ncontig < 0 ||
      (ncontig > 0 && !order) || !cum || nentries < 0 || (nentries > 0 && !entries) ||
      cum[(1 << 24) - 1] != nentries)
    return PGA_ERR_ARG;
  const int eb = 9 + post_bytes + cont_bytes;
  std::vector<int64_t> inv(ncontig);          // contig -> its place in the order
  for (int i = 0; i < ncontig; i++) {
    if (order[i] < 0 || order[i] >= ncontig) return PGA_ERR_ARG;
    inv[order[i]] = i;
  }
  const uint64_t sign = (uint64_t)1 << (8 * cont_bytes - 1);
  std::string s(stem);
  const size_t slash = s.rfind('/');
  const std::string dir = slash == std::string::npos ? "." : s.substr(0, slash);
  const std::string root = slash == std::string::npos ? s : s.substr(slash + 1);

  // parts: whole panels, about nentries / nparts entries each
  std::vector<int64_t> pstart(NPANEL + 1, 0);  // first entry of each panel
  for (int q = 1; q <= NPANEL; q++) pstart[q] = cum[((int64_t)q << PANEL_SHIFT) - 1];
  std::vector<int> split(nparts + 1, NPANEL);
  split[0] = 0;
  for (int p = 1, q = 0; p < nparts; p++) {
    const int64_t want = nentries * p / nparts;
    while (q < NPANEL && pstart[q] < want) q++;
    split[p] = std::max(q, split[p - 1]);
  }

  std::vector<uint8_t> buf;
  for (int p = 0; p < nparts; p++) {
    const int64_t a = pstart[split[p]], b = pstart[split[p + 1]];
    const std::string path = dir + "/." + root + ".ktab." + std::to_string(p + 1);
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return PGA_ERR_ARG;
    const int k = GIX_KMER;
    const int64_t n = b - a;
    bool ok = put(f, &k, sizeof(int)) && put(f, &n, sizeof(int64_t));
    int first_panel = split[p];
    while (first_panel < NPANEL && pstart[first_panel + 1] == pstart[first_panel]) first_panel++;
    for (int64_t i0 = a; ok && i0 < b; i0 += 1 << 16) {
      const int64_t i1 = std::min(b, i0 + ((int64_t)1 << 16));
      buf.assign(entries + i0 * eb, entries + i1 * eb);
      for (int64_t i = i0; i < i1; i++) {
        uint8_t *e = buf.data() + (i - i0) * eb;
        uint64_t cs = 0;
        for (int q = 0; q < cont_bytes; q++) cs |= (uint64_t)e[9 + post_bytes + q] << (8 * q);
        const uint64_t c = cs & (sign - 1);
        if ((int64_t)c >= ncontig) return PGA_ERR_ARG;
        cs = (uint64_t)inv[c] | (cs & sign);
        for (int q = 0; q < cont_bytes; q++) e[9 + post_bytes + q] = (uint8_t)(cs >> (8 * q));
        if (i == a) e[8] = first_panel == split[p] ? 0 : (uint8_t)panel_lcp(first_panel, split[p]);
      }
      ok = put(f, buf.data(), buf.size());
    }
    if (fclose(f) != 0) ok = false;
    if (!ok) return PGA_ERR_ARG;
  }

  const std::string path = dir + "/" + root + ".gix";
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) return PGA_ERR_ARG;
  const int k = GIX_KMER, one = 1, three = 3, freq = 0;
  const int64_t end = -1;
  bool ok = put(f, &k, sizeof(int)) && put(f, &nparts, sizeof(int)) && put(f, &one, sizeof(int)) &&
            put(f, &three, sizeof(int)) && put(f, cum, sizeof(int64_t) << 24) &&
            put(f, &post_bytes, sizeof(int)) && put(f, &cont_bytes, sizeof(int)) && put(f, &nparts, sizeof(int)) &&
            put(f, &largest, sizeof(int64_t)) && put(f, &freq, sizeof(int)) && put(f, &ncontig, sizeof(int)) &&
            (ncontig == 0 || put(f, order, sizeof(int32_t) * (size_t)ncontig)) && put(f, &end, sizeof(int64_t));
  if (fclose(f) != 0) ok = false;
  return ok ? PGA_OK : PGA_ERR_ARG;
}

namespace {

bool get(FILE *f, void *p, size_t n) { return fread(p, 1, n, f) == n; }

// Bases two k-mers share from the start; a k-mer is its 3 prefix bytes (the
// entry's place in the 2^24 table) and the entry's 7 suffix bytes.
int kmer_lcp(uint32_t pa, const uint8_t *sa, uint32_t pb, const uint8_t *sb) {
  uint8_t a[10], b[10];
  a[0] = (uint8_t)(pa >> 16), a[1] = (uint8_t)(pa >> 8), a[2] = (uint8_t)pa;
  b[0] = (uint8_t)(pb >> 16), b[1] = (uint8_t)(pb >> 8), b[2] = (uint8_t)pb;
  memcpy(a + 3, sa, 7);
  memcpy(b + 3, sb, 7);
  for (int i = 0; i < 10; i++)
    if (a[i] != b[i]) {
      int z = 0;
      while (z < 3 && !((a[i] ^ b[i]) & (0xc0 >> (2 * z)))) z++;
      return 4 * i + z;
    }
  return GIX_KMER;
}

}  // namespace

extern "C" int pga_read_gix(const char *stem, int *hdr6, int32_t *order, int64_t order_cap, int64_t *cum,
                            int64_t *largest, int64_t *nentries, uint8_t *entries, int64_t entries_cap) {
  if (!stem || !hdr6 || !largest || !nentries) return PGA_ERR_ARG;
  std::string s(stem);
  const size_t slash = s.rfind('/');
  const std::string dir = slash == std::string::npos ? "." : s.substr(0, slash);
  const std::string root = slash == std::string::npos ? s : s.substr(slash + 1);

  FILE *f = fopen((dir + "/" + root + ".gix").c_str(), "rb");
  if (!f) return PGA_ERR_ARG;
  int head[4], pc[3], freq = 0, nctg = 0;
  std::vector<int64_t> table((size_t)1 << 24);
  int64_t big = 0, end = 0;
  bool ok = get(f, head, sizeof(head)) && get(f, table.data(), sizeof(int64_t) << 24) && get(f, pc, sizeof(pc)) &&
            get(f, &big, sizeof(big)) && get(f, &freq, sizeof(int)) && get(f, &nctg, sizeof(int));
  std::vector<int32_t> ord;
  if (ok && nctg >= 0 && nctg <= (1 << 30)) {
    ord.resize((size_t)nctg);
    ok = (nctg == 0 || get(f, ord.data(), sizeof(int32_t) * (size_t)nctg)) && get(f, &end, sizeof(end));
  } else {
    ok = false;
  }
  fclose(f);
  const int nparts = head[1], post_bytes = pc[0], cont_bytes = pc[1];
  if (!ok || head[0] != GIX_KMER || nparts < 1 || nparts > NPANEL || pc[2] != nparts || post_bytes < 1 ||
      post_bytes > 8 || cont_bytes < 1 || cont_bytes > 8 || end != -1)
    return PGA_ERR_ARG;
  std::vector<char> seen((size_t)nctg, 0);
  for (int i = 0; i < nctg; i++) {
    if (ord[(size_t)i] < 0 || ord[(size_t)i] >= nctg || seen[(size_t)ord[(size_t)i]]) return PGA_ERR_ARG;
    seen[(size_t)ord[(size_t)i]] = 1;
  }
  const int64_t n = table[((size_t)1 << 24) - 1];
  hdr6[0] = GIX_KMER, hdr6[1] = nparts, hdr6[2] = post_bytes, hdr6[3] = cont_bytes, hdr6[4] = freq,
  hdr6[5] = nctg;
  *largest = big;
  *nentries = n;
  if (!entries) return PGA_OK;  // sizes only
  if (entries_cap < n || !cum || (nctg > 0 && (!order || order_cap < nctg))) return PGA_ERR_ARG;
  std::copy(table.begin(), table.end(), cum);
  std::copy(ord.begin(), ord.end(), order);

  // the parts, back to back; contigs renumbered from places in the order
  const int eb = 9 + post_bytes + cont_bytes;
  const uint64_t sign = (uint64_t)1 << (8 * cont_bytes - 1);
  int64_t at = 0;
  std::vector<int64_t> part_start;
  for (int p = 1; p <= nparts; p++) {
    FILE *g = fopen((dir + "/." + root + ".ktab." + std::to_string(p)).c_str(), "rb");
    if (!g) return PGA_ERR_ARG;
    int k = 0;
    int64_t m = -1;
    bool pok = get(g, &k, sizeof(int)) && get(g, &m, sizeof(int64_t)) && k == GIX_KMER && m >= 0 && at + m <= n &&
               (m == 0 || get(g, entries + at * eb, (size_t)(m * eb)));
    fclose(g);
    if (!pok) return PGA_ERR_ARG;
    part_start.push_back(at);
    at += m;
  }
  if (at != n) return PGA_ERR_ARG;
  for (int64_t i = 0; i < n; i++) {
    uint8_t *e = entries + i * eb;
    uint64_t cs = 0;
    for (int q = 0; q < cont_bytes; q++) cs |= (uint64_t)e[9 + post_bytes + q] << (8 * q);
    const uint64_t place = cs & (sign - 1);
    if ((int64_t)place >= nctg) return PGA_ERR_ARG;
    cs = (uint64_t)ord[(size_t)place] | (cs & sign);
    for (int q = 0; q < cont_bytes; q++) e[9 + post_bytes + q] = (uint8_t)(cs >> (8 * q));
  }
  // a part's first entry: its LCP to the entry before it (the index's first: 0)
  uint32_t pfx = 0;
  for (int64_t ps : part_start) {
    if (ps >= n) continue;
    if (ps == 0) {
      entries[8] = 0;
      continue;
    }
    while (pfx < ((uint32_t)1 << 24) && table[pfx] <= ps - 1) pfx++;
    const uint32_t pa = pfx;  // prefix of entry ps - 1
    uint32_t pb = pa;
    while (pb < ((uint32_t)1 << 24) && table[pb] <= ps) pb++;
    entries[ps * eb + 8] = (uint8_t)kmer_lcp(pa, entries + (ps - 1) * eb, pb, entries + ps * eb);
  }
  return PGA_OK;
}
