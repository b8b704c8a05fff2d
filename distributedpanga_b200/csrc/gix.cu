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
