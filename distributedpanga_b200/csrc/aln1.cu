// The .1aln output of the alignment path: la_merge's file
// (src/fastga_pipeline.c:1616-1656) written as a ONE file, in either of ONE's
// encodings: ASCII (pga_write_1aln) or binary (pga_write_1aln_binary, the
// encoding the reference's open_Aln_Write asks ONElib for,
// lib/alncode.c:239-270).  Both carry the header (file type "aln",
// provenance, references, the line definitions), the trace spacing line, the
// GDB skeleton (Write_Skeleton, lib/GDB.c:2059-2086) and one alignment per
// record in la_sort order (Write_Aln_Overlap / Write_Aln_Trace,
// lib/alncode.c:272-305):
//
//   A aread abpos aepos bread bbpos bepos
//   R                               (b reverse-complemented)
//   D diffs
//   T n b-delta per trace interval
//   X n differences per trace interval
//
// Host code only; it needs no GPU.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <memory>
#include <string>
#include <vector>
#include "../../include/pga_b200.h"

namespace {

// ONE format version this file declares (the reader checks the major).
constexpr int ONE_MAJOR = 2, ONE_MINOR = 1;

// The "aln" file type's line definitions, in their schema order
// (lib/alncode.c:19-52): O = object line, D = data line, G = the preceding
// object groups this object type; then the field types.  An ASCII ONE file
// carries them in its header ('~' lines) so that its counts and records
// parse.
const char *const ALN_SCHEMA[] = {
    "D t 1 3 INT",
    "O g 0",
    "G S 0",
    "O S 1 6 STRING",
    "D G 1 3 INT",
    "D C 1 3 INT",
    "O a 0",
    "G A 0",
    "D p 2 3 INT 3 INT",
    "O A 6 3 INT 3 INT 3 INT 3 INT 3 INT 3 INT",
    "D L 2 3 INT 3 INT",
    "D R 0",
    "D D 1 3 INT",
    "D T 1 8 INT_LIST",
    "D X 1 8 INT_LIST",
    "D Q 1 3 INT",
    "D E 1 3 INT",
    "D Z 1 6 STRING",
    "D U 1 3 INT",
};

void put_string(FILE *f, const char *s) { fprintf(f, " %zu %s", strlen(s), s); }

bool bad_args(const char *path, const char *program, const char *version, const char *command, const char *db_name,
              int tspace, int nscaff, const char *const *scaff_name, const int64_t *scaff_len,
              const int32_t *scaff_fctg, const int64_t *contig_sbeg, const int64_t *contig_len, int64_t nalign,
              const int32_t *recs9, const int64_t *trace_off, const uint8_t *trace) {
  if (!path || !program || !version || !command || !db_name || tspace <= 0 || nscaff < 0 || nalign < 0 ||
      (nscaff > 0 && (!scaff_name || !scaff_len || !scaff_fctg || !contig_sbeg || !contig_len)) ||
      (nalign > 0 && (!recs9 || !trace_off || !trace)))
    return true;
  for (int s = 0; s < nscaff; s++)
    if (!scaff_name[s] || strchr(scaff_name[s], '\n') || scaff_fctg[s + 1] < scaff_fctg[s]) return true;
  for (int64_t i = 0; i < nalign; i++)
    if (recs9[9 * i + 8] < 0) return true;
  return false;
}

// What both encodings write first: the version line, provenance (with the
// local time), the references (the GDB as 1, the working directory as 3) and
// the line definitions.
void write_head(FILE *f, const char *program, const char *version, const char *command, const char *db_name,
                const char *cwd) {
  char date[64];
  time_t now = time(nullptr);
  struct tm tmv;
  localtime_r(&now, &tmv);
  strftime(date, sizeof(date), "%F_%T", &tmv);
  fprintf(f, "1 3 aln %d %d", ONE_MAJOR, ONE_MINOR);
  fprintf(f, "\n! 4");
  put_string(f, program);
  put_string(f, version);
  put_string(f, command);
  put_string(f, date);
  fprintf(f, "\n.");
  fprintf(f, "\n<");
  put_string(f, db_name);
  fprintf(f, " 1");
  if (cwd) {
    fprintf(f, "\n<");
    put_string(f, cwd);
    fprintf(f, " 3");
  }
  fprintf(f, "\n.");
  for (const char *d : ALN_SCHEMA) fprintf(f, "\n~ %s", d);
}

// ---- ONE's binary encoding (lib/ONElib.c: writeHeader, oneWriteLine,
// oneWriteFooter, as its reader oneFileOpenRead / oneReadLine takes them).
//
// After the line definitions the header ends with "$ <big-endian>" and the
// data lines follow, each one byte of line code and then its fields with no
// separator: integers as variable-length integers (below), a character as
// its byte, a string or list as its length (an integer) and then its
// contents -- a string's bytes, or an integer list's first value followed
// by the byte width w of its successive differences and each difference in
// w little-endian bytes.  A '\n' where a line would start ends the data.
// The footer follows it: per line type with lines, its count ("# t n"),
// its largest and total list length ("@", "+"), per object type the largest
// number of lines and list total of each type it contains ("% t # u n",
// "% t + u n"), and the byte offset of every object as an index line ("&":
// the type, then offset 0 = the data's start and offset i = object i's
// line).  "^\n" ends it, and the file's last 8 bytes are the footer's offset.
//
// The line code is 0x80 | c << 1, c = 0-25 for 'A'-'Z', 26-51 for 'a'-'z',
// 52 for a list codec line ';' and 53 for '&'.  Bit 0 set says the line's
// list is coded with its type's list codec: the number of bits, then the
// coded bytes.  The codec is a ';' line of the footer (the type, then the
// serialized codec as a string).  ONElib builds one from a type's first
// 100,000 list bytes and codes every later list; here the trace lists' codec
// is built from all of them, and a list is coded where that is shorter.
// Readers decode per line, either way.
uint8_t line_code(char t) {
  int c = (t >= 'A' && t <= 'Z') ? t - 'A' : (t >= 'a' && t <= 'z') ? 26 + t - 'a' : t == ';' ? 52 : 53;
  return (uint8_t)(0x80 | (c << 1));
}

// Variable-length integer: 0..63 and -64..-1 in one byte (0x40 | v, and the
// value's own low byte, whose bits 6 and 7 are set); 64..8191 in two (0x20 |
// v >> 8, then v's low byte); otherwise a tag byte (k - 1 for a value >= 0,
// 0x80 | (k - 1) below 0) and the value's k low bytes, little-endian, k the
// fewest of 2..8 that hold it (sign-extended on reading).
int ltf(uint8_t *u, int64_t v) {
  if (v >= -64 && v < 64) {
    u[0] = (uint8_t)((uint64_t)v & 0xff) | 0x40;
    return 1;
  }
  if (v >= 64 && v < 8192) {
    u[0] = (uint8_t)(0x20 | (v >> 8));
    u[1] = (uint8_t)(v & 0xff);
    return 2;
  }
  const uint64_t m = v >= 0 ? (uint64_t)v : ~(uint64_t)v;
  int k = 2;
  while (k < 8 && (m >> (8 * k)) != 0) k++;
  u[0] = (uint8_t)((v >= 0 ? 0 : 0x80) | (k - 1));
  for (int b = 0; b < k; b++) u[1 + b] = (uint8_t)((uint64_t)v >> (8 * b));
  return 1 + k;
}

// An integer list's bytes after its first value: the width w (1..8) of its
// successive differences, and each difference's w low bytes, little-endian
// (sign-extended on reading).  w is the fewest bytes that hold every
// difference with its sign bit.
int compact_diffs(const int64_t *v, int64_t n, std::vector<uint8_t> &out) {
  uint64_t m = 0;
  for (int64_t i = 1; i < n; i++) {
    const int64_t d = v[i] - v[i - 1];
    m |= d >= 0 ? (uint64_t)d : ~(uint64_t)d;
  }
  int w = 1;
  for (m >>= 7; w < 8 && m != 0; m >>= 8) w++;
  out.clear();
  for (int64_t i = 1; i < n; i++) {
    const uint64_t d = (uint64_t)(v[i] - v[i - 1]);
    for (int b = 0; b < w; b++) out.push_back((uint8_t)(d >> (8 * b)));
  }
  return w;
}

// A line type's list codec: a prefix code over bytes with codes of at most
// CODE_MAX bits, in the form ONE readers take (vcDeserialize / vcDecode,
// lib/ONElib.c:3338-3735).  The code lengths are the optimal ones under
// that limit, by package-merge (Larmore & Hirschberg, J. ACM 37(3), 1990)
// over the byte histogram of all the type's lists; codes are canonical
// (by length, then byte).  Every byte that occurs has a code, so there is
// no escape code.
struct ListCodec {
  static constexpr int CODE_MAX = 12;
  uint8_t len[256] = {};
  uint16_t bits[256] = {};

  explicit ListCodec(const uint64_t *hist) {
    std::vector<int> sym;
    for (int s = 0; s < 256; s++)
      if (hist[s]) sym.push_back(s);
    const int n = (int)sym.size();
    if (n == 0) return;
    if (n == 1) {
      len[sym[0]] = 1;
    } else {
      std::stable_sort(sym.begin(), sym.end(), [&](int a, int b) { return hist[a] < hist[b]; });
      // items: a weight and how often each symbol (by rank) is in it
      struct Item {
        uint64_t w;
        std::vector<uint16_t> c;
      };
      std::vector<Item> leaves((size_t)n), cur;
      for (int i = 0; i < n; i++) {
        leaves[(size_t)i].w = hist[sym[(size_t)i]];
        leaves[(size_t)i].c.assign((size_t)n, 0);
        leaves[(size_t)i].c[(size_t)i] = 1;
      }
      cur = leaves;
      for (int level = 1; level < CODE_MAX; level++) {
        std::vector<Item> pk;
        for (size_t k = 0; k + 1 < cur.size(); k += 2) {
          Item p{cur[k].w + cur[k + 1].w, cur[k].c};
          for (int i = 0; i < n; i++) p.c[(size_t)i] += cur[k + 1].c[(size_t)i];
          pk.push_back(std::move(p));
        }
        std::vector<Item> next;
        size_t a = 0, b = 0;
        while (a < leaves.size() || b < pk.size())
          if (b >= pk.size() || (a < leaves.size() && leaves[a].w <= pk[b].w))
            next.push_back(leaves[a++]);
          else
            next.push_back(std::move(pk[b++]));
        cur = std::move(next);
      }
      for (size_t k = 0; k < (size_t)(2 * n - 2); k++)
        for (int i = 0; i < n; i++) len[sym[(size_t)i]] = (uint8_t)(len[sym[(size_t)i]] + cur[k].c[(size_t)i]);
    }
    std::vector<int> order;
    for (int s = 0; s < 256; s++)
      if (len[s]) order.push_back(s);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return len[a] < len[b]; });
    uint32_t code = 0;
    int prev = len[order[0]];
    for (int s : order) {
      code <<= (len[s] - prev);
      prev = len[s];
      bits[s] = (uint16_t)code++;
    }
  }

  // vcSerialize's layout: big-endian flag, escape code and its length (two
  // ints), then per byte its code length and, where nonzero, its code.
  std::vector<uint8_t> serial() const {
    std::vector<uint8_t> o;
    o.push_back(0);
    const int32_t esc = -1, elen = 0;
    for (int32_t v : {esc, elen})
      for (int b = 0; b < 4; b++) o.push_back((uint8_t)((uint32_t)v >> (8 * b)));
    for (int s = 0; s < 256; s++) {
      o.push_back(len[s]);
      if (len[s]) {
        o.push_back((uint8_t)(bits[s] & 0xff));
        o.push_back((uint8_t)(bits[s] >> 8));
      }
    }
    return o;
  }

  // The coded form of in (vcEncode's): a bit stream of two flag bits (0 0:
  // written little-endian) and the bytes' codes, cut into 64-bit words
  // whose first bit is the most significant; each whole word stored as a
  // little-endian integer, the last part word's bytes most significant
  // first, and, when there is a whole word, the file's bytes 0 and 7
  // exchanged so that the flag bits come first.  Returns the bit count.
  int64_t encode(const std::vector<uint8_t> &in, std::vector<uint8_t> &out) const {
    std::vector<uint64_t> words;
    uint64_t cur = 0;
    int used = 0;
    int64_t nbits = 0;
    auto put = [&](uint32_t c, int l) {
      nbits += l;
      if (used + l <= 64) {
        cur |= (uint64_t)c << (64 - used - l);
        used += l;
      } else {
        const int r = used + l - 64;
        cur |= (uint64_t)c >> r;
        words.push_back(cur);
        cur = (uint64_t)c << (64 - r);
        used = r;
      }
      if (used == 64) {
        words.push_back(cur);
        cur = 0;
        used = 0;
      }
    };
    put(0, 2);
    for (uint8_t x : in) put(bits[x], len[x]);
    out.clear();
    for (uint64_t w : words)
      for (int b = 0; b < 8; b++) out.push_back((uint8_t)(w >> (8 * b)));
    for (int k = 0; k < (used + 7) / 8; k++) out.push_back((uint8_t)(cur >> (56 - 8 * k)));
    if (!words.empty()) std::swap(out[0], out[7]);
    return nbits;
  }
};

// Trace lists are coded only when their compacted bytes reach this many
// (below it the codec's own ~300 bytes would not pay).
constexpr uint64_t CODEC_MIN_BYTES = 4096;

class BinOut {
 public:
  BinOut(FILE *f, int64_t pos) : f_(f), pos_(pos) { buf_.reserve(CHUNK + 4096); }
  int64_t pos() const { return pos_ + (int64_t)buf_.size(); }
  void byte(uint8_t b) {
    buf_.push_back(b);
    spill();
  }
  void bytes(const void *p, size_t n) {
    const uint8_t *c = (const uint8_t *)p;
    buf_.insert(buf_.end(), c, c + n);
    spill();
  }
  void integer(int64_t v) {
    uint8_t u[9];
    bytes(u, (size_t)ltf(u, v));
  }
  // an uncoded integer list of n >= 1 values, after its length
  void int_list(const int64_t *v, int64_t n) {
    integer(v[0]);
    if (n == 1) return;
    const int w = compact_diffs(v, n, tmp_);
    byte((uint8_t)w);
    bytes(tmp_.data(), tmp_.size());
  }
  // footer text lines: "k t v" for k = '#' count, '@' largest list, '+'
  // list total; "% t k u v" for object type t's largest count (k '#') or
  // list total (k '+') of line type u within one object
  void count(char k, char t, int64_t v) {
    char line[64];
    const int n = snprintf(line, sizeof(line), "%c %c %lld\n", k, t, (long long)v);
    bytes(line, (size_t)n);
  }
  void stat(char t, char k, char u, int64_t v) {
    char line[64];
    const int n = snprintf(line, sizeof(line), "%% %c %c %c %lld\n", t, k, u, (long long)v);
    bytes(line, (size_t)n);
  }
  bool flush() {
    if (!buf_.empty() && fwrite(buf_.data(), 1, buf_.size(), f_) != buf_.size()) return false;
    pos_ += (int64_t)buf_.size();
    buf_.clear();
    return true;
  }
  bool ok() const { return ok_; }

 private:
  static constexpr size_t CHUNK = 1 << 20;
  void spill() {
    if (buf_.size() >= CHUNK) ok_ = flush() && ok_;
  }
  FILE *f_;
  int64_t pos_;
  std::vector<uint8_t> buf_, tmp_;
  bool ok_ = true;
};

}  // namespace

extern "C" int pga_write_1aln(const char *path, const char *program, const char *version, const char *command,
                              const char *db_name, const char *cwd, int tspace, int nscaff,
                              const char *const *scaff_name, const int64_t *scaff_len, const int32_t *scaff_fctg,
                              const int64_t *contig_sbeg, const int64_t *contig_len, int64_t nalign,
                              const int32_t *recs9, const int64_t *trace_off, const uint8_t *trace) {
  if (bad_args(path, program, version, command, db_name, tspace, nscaff, scaff_name, scaff_len, scaff_fctg,
               contig_sbeg, contig_len, nalign, recs9, trace_off, trace))
    return PGA_ERR_ARG;
  FILE *f = fopen(path, "w");
  if (!f) return PGA_ERR_ARG;

  // header, then the object counts readers use
  int64_t tmax = 0, ttot = 0;
  for (int64_t i = 0; i < nalign; i++) {
    int64_t n = recs9[9 * i + 8] / 2;
    if (n > tmax) tmax = n;
    ttot += n;
  }
  write_head(f, program, version, command, db_name, cwd);
  fprintf(f, "\n.");
  fprintf(f, "\n# g %d", nscaff > 0 ? 1 : 0);
  fprintf(f, "\n# S %d", nscaff);
  fprintf(f, "\n# A %lld", (long long)nalign);
  if (nalign > 0) {
    fprintf(f, "\n# T %lld\n@ T %lld\n+ T %lld", (long long)nalign, (long long)tmax, (long long)ttot);
    fprintf(f, "\n# X %lld\n@ X %lld\n+ X %lld", (long long)nalign, (long long)tmax, (long long)ttot);
  }
  fprintf(f, "\n.");

  // trace spacing
  fprintf(f, "\nt %d", tspace);

  // GDB skeleton: per scaffold its name, then gaps and contigs in order
  if (nscaff > 0) {
    fprintf(f, "\ng");
    for (int s = 0; s < nscaff; s++) {
      fprintf(f, "\nS");
      put_string(f, scaff_name[s]);
      int64_t spos = 0;
      for (int32_t c = scaff_fctg[s]; c < scaff_fctg[s + 1]; c++) {
        if (contig_sbeg[c] > spos) fprintf(f, "\nG %lld", (long long)(contig_sbeg[c] - spos));
        fprintf(f, "\nC %lld", (long long)contig_len[c]);
        spos = contig_sbeg[c] + contig_len[c];
      }
      if (scaff_len[s] > spos) fprintf(f, "\nG %lld", (long long)(scaff_len[s] - spos));
    }
  }

  // alignments
  for (int64_t i = 0; i < nalign; i++) {
    const int32_t *r = recs9 + 9 * i;
    const uint8_t *tr = trace + trace_off[i];
    const int tlen = r[8];
    fprintf(f, "\nA %d %d %d %d %d %d", r[0], r[1], r[2], r[3], r[4], r[5]);
    if (r[6]) fprintf(f, "\nR");
    fprintf(f, "\nD %d", r[7]);
    fprintf(f, "\nT %d", tlen / 2);
    for (int x = 1; x < tlen; x += 2) fprintf(f, " %d", tr[x]);
    fprintf(f, "\nX %d", tlen / 2);
    for (int x = 0; x < tlen; x += 2) fprintf(f, " %d", tr[x]);
  }
  fprintf(f, "\n");
  int bad = ferror(f);
  if (fclose(f) != 0) bad = 1;
  return bad ? PGA_ERR_ARG : PGA_OK;
}

extern "C" int pga_write_1aln_binary(const char *path, const char *program, const char *version,
                                     const char *command, const char *db_name, const char *cwd, int tspace,
                                     int nscaff, const char *const *scaff_name, const int64_t *scaff_len,
                                     const int32_t *scaff_fctg, const int64_t *contig_sbeg,
                                     const int64_t *contig_len, int64_t nalign, const int32_t *recs9,
                                     const int64_t *trace_off, const uint8_t *trace) {
  if (bad_args(path, program, version, command, db_name, tspace, nscaff, scaff_name, scaff_len, scaff_fctg,
               contig_sbeg, contig_len, nalign, recs9, trace_off, trace))
    return PGA_ERR_ARG;
  FILE *f = fopen(path, "wb");
  if (!f) return PGA_ERR_ARG;
  write_head(f, program, version, command, db_name, cwd);
  fprintf(f, "\n$ 0\n");  // little-endian; the data start after this line
  const int64_t start = (int64_t)ftello(f);
  if (start < 0) {
    fclose(f);
    return PGA_ERR_ARG;
  }
  BinOut o(f, start);

  // the footer's figures, gathered as the lines go out
  std::vector<int64_t> ix_g{start}, ix_S{start}, ix_A{start};
  int64_t nG = 0, nC = 0, nR = 0, smax = 0, stot = 0, sC = 0, sG = 0, tmax = 0, ttot = 0;

  o.byte(line_code('t'));
  o.integer(tspace);

  // GDB skeleton
  if (nscaff > 0) {
    ix_g.push_back(o.pos());
    o.byte(line_code('g'));
    for (int s = 0; s < nscaff; s++) {
      ix_S.push_back(o.pos());
      const int64_t len = (int64_t)strlen(scaff_name[s]);
      o.byte(line_code('S'));
      o.integer(len);
      o.bytes(scaff_name[s], (size_t)len);
      smax = len > smax ? len : smax;
      stot += len;
      int64_t spos = 0, cG = 0, cC = 0;
      for (int32_t c = scaff_fctg[s]; c < scaff_fctg[s + 1]; c++) {
        if (contig_sbeg[c] > spos) {
          o.byte(line_code('G'));
          o.integer(contig_sbeg[c] - spos);
          cG++;
        }
        o.byte(line_code('C'));
        o.integer(contig_len[c]);
        cC++;
        spos = contig_sbeg[c] + contig_len[c];
      }
      if (scaff_len[s] > spos) {
        o.byte(line_code('G'));
        o.integer(scaff_len[s] - spos);
        cG++;
      }
      nG += cG;
      nC += cC;
      sG = cG > sG ? cG : sG;
      sC = cC > sC ? cC : sC;
    }
  }

  // alignments
  // the trace lists' codecs (T: b-deltas, the odd trace bytes; X: diffs, the
  // even ones), from the byte histogram of all their compacted lists
  std::vector<int64_t> list;
  std::vector<uint8_t> raw, enc;
  auto trace_list = [&](const uint8_t *tr, int64_t n, int pass) {
    list.resize((size_t)n);
    for (int64_t x = 0; x < n; x++) list[(size_t)x] = tr[2 * x + (pass ? 0 : 1)];
  };
  std::unique_ptr<ListCodec> codec[2];
  {
    uint64_t hist[2][256] = {};
    uint64_t total[2] = {0, 0};
    for (int64_t i = 0; i < nalign; i++) {
      const int64_t n = recs9[9 * i + 8] / 2;
      if (n < 2) continue;
      for (int pass = 0; pass < 2; pass++) {
        trace_list(trace + trace_off[i], n, pass);
        compact_diffs(list.data(), n, raw);
        for (uint8_t x : raw) hist[pass][x]++;
        total[pass] += raw.size();
      }
    }
    for (int pass = 0; pass < 2; pass++)
      if (total[pass] >= CODEC_MIN_BYTES) codec[pass].reset(new ListCodec(hist[pass]));
  }

  ix_A.reserve((size_t)nalign + 1);
  for (int64_t i = 0; i < nalign; i++) {
    const int32_t *r = recs9 + 9 * i;
    const uint8_t *tr = trace + trace_off[i];
    const int64_t n = r[8] / 2;
    ix_A.push_back(o.pos());
    o.byte(line_code('A'));
    for (int k = 0; k < 6; k++) o.integer(r[k]);
    if (r[6]) {
      o.byte(line_code('R'));
      nR++;
    }
    o.byte(line_code('D'));
    o.integer(r[7]);
    for (int pass = 0; pass < 2; pass++) {
      trace_list(tr, n, pass);
      int w = 0;
      int64_t nbits = 0;
      bool coded = false;
      if (n >= 2) {
        w = compact_diffs(list.data(), n, raw);
        if (codec[pass]) {
          uint8_t u[9];
          nbits = codec[pass]->encode(raw, enc);
          coded = ltf(u, nbits) + enc.size() < raw.size();
        }
      }
      o.byte((uint8_t)(line_code(pass ? 'X' : 'T') | (coded ? 1 : 0)));
      o.integer(n);
      if (n == 0) continue;
      o.integer(list[0]);
      if (n == 1) continue;
      o.byte((uint8_t)w);
      if (coded) {
        o.integer(nbits);
        o.bytes(enc.data(), enc.size());
      } else {
        o.bytes(raw.data(), raw.size());
      }
    }
    tmax = n > tmax ? n : tmax;
    ttot += n;
  }
  o.byte('\n');  // end of data

  // footer, in the line definitions' order
  const int64_t foot = o.pos();
  auto index = [&](char t, const std::vector<int64_t> &ix) {
    o.byte(line_code('&'));
    o.byte((uint8_t)t);
    o.integer((int64_t)ix.size());
    o.int_list(ix.data(), (int64_t)ix.size());
  };
  o.count('#', 't', 1);
  if (nscaff > 0) {
    o.count('#', 'g', 1);
    if (nC) o.stat('g', '#', 'C', nC);
    if (nG) o.stat('g', '#', 'G', nG);
    o.stat('g', '#', 'S', nscaff);
    if (stot) o.stat('g', '+', 'S', stot);
    index('g', ix_g);
    o.count('#', 'S', nscaff);
    if (smax) o.count('@', 'S', smax);
    if (stot) o.count('+', 'S', stot);
    if (sC) o.stat('S', '#', 'C', sC);
    if (sG) o.stat('S', '#', 'G', sG);
    index('S', ix_S);
    if (nG) o.count('#', 'G', nG);
    if (nC) o.count('#', 'C', nC);
  }
  if (nalign > 0) {
    o.count('#', 'A', nalign);
    o.stat('A', '#', 'D', 1);
    if (nR) o.stat('A', '#', 'R', 1);
    o.stat('A', '#', 'T', 1);
    if (tmax) o.stat('A', '+', 'T', tmax);
    o.stat('A', '#', 'X', 1);
    if (tmax) o.stat('A', '+', 'X', tmax);
    index('A', ix_A);
    if (nR) o.count('#', 'R', nR);
    o.count('#', 'D', nalign);
    for (int pass = 0; pass < 2; pass++) {
      const char t = pass ? 'X' : 'T';
      o.count('#', t, nalign);
      if (tmax) o.count('@', t, tmax);
      if (ttot) o.count('+', t, ttot);
      if (codec[pass]) {
        const std::vector<uint8_t> ser = codec[pass]->serial();
        o.byte(line_code(';'));
        o.byte((uint8_t)t);
        o.integer((int64_t)ser.size());
        o.bytes(ser.data(), ser.size());
      }
    }
  }
  o.bytes("^\n", 2);
  uint8_t off8[8];
  for (int b = 0; b < 8; b++) off8[b] = (uint8_t)((uint64_t)foot >> (8 * b));
  o.bytes(off8, 8);
  bool good = o.ok() && o.flush();
  good = !ferror(f) && good;
  if (fclose(f) != 0) good = false;
  return good ? PGA_OK : PGA_ERR_ARG;
}
