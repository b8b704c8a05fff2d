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
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
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
// The line code is 0x80 | c << 1, c = 0-25 for 'A'-'Z', 26-51 for 'a'-'z'
// and 53 for '&'.  Bit 0 set says the line's list is Huffman-coded with a
// codec trained on the file's earlier lists (ONElib switches to one after
// 100,000 list bytes); it stays clear here, every list is written as it is,
// and readers decode either per line.
uint8_t line_code(char t) {
  int c = (t >= 'A' && t <= 'Z') ? t - 'A' : (t >= 'a' && t <= 'z') ? 26 + t - 'a' : 53;
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
  // an integer list of n >= 1 values, after its length
  void int_list(const int64_t *v, int64_t n) {
    integer(v[0]);
    if (n == 1) return;
    uint64_t m = 0;
    for (int64_t i = 1; i < n; i++) {
      const int64_t d = v[i] - v[i - 1];
      m |= d >= 0 ? (uint64_t)d : ~(uint64_t)d;
    }
    int w = 1;
    for (m >>= 7; w < 8 && m != 0; m >>= 8) w++;
    byte((uint8_t)w);
    for (int64_t i = 1; i < n; i++) {
      const uint64_t d = (uint64_t)(v[i] - v[i - 1]);
      for (int b = 0; b < w; b++) buf_.push_back((uint8_t)(d >> (8 * b)));
      spill();
    }
  }
  void text(const char *fmt, long long a, long long b = 0) {
    char line[96];
    const int n = snprintf(line, sizeof(line), fmt, a, b);
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
  std::vector<uint8_t> buf_;
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
  std::vector<int64_t> list;
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
    list.resize((size_t)n);
    for (int pass = 0; pass < 2; pass++) {  // T: b-deltas (odd bytes), X: diffs (even bytes)
      o.byte(line_code(pass ? 'X' : 'T'));
      o.integer(n);
      if (n == 0) continue;
      for (int64_t x = 0; x < n; x++) list[(size_t)x] = tr[2 * x + (pass ? 0 : 1)];
      o.int_list(list.data(), n);
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
  o.text("# t %lld\n", 1);
  if (nscaff > 0) {
    o.text("# g %lld\n", 1);
    if (nC) o.text("%% g # C %lld\n", nC);
    if (nG) o.text("%% g # G %lld\n", nG);
    o.text("%% g # S %lld\n", nscaff);
    if (stot) o.text("%% g + S %lld\n", stot);
    index('g', ix_g);
    o.text("# S %lld\n", nscaff);
    if (smax) o.text("@ S %lld\n", smax);
    if (stot) o.text("+ S %lld\n", stot);
    if (sC) o.text("%% S # C %lld\n", sC);
    if (sG) o.text("%% S # G %lld\n", sG);
    index('S', ix_S);
    if (nG) o.text("# G %lld\n", nG);
    if (nC) o.text("# C %lld\n", nC);
  }
  if (nalign > 0) {
    o.text("# A %lld\n", nalign);
    o.text("%% A # D %lld\n", 1);
    if (nR) o.text("%% A # R %lld\n", 1);
    o.text("%% A # T %lld\n", 1);
    if (tmax) o.text("%% A + T %lld\n", tmax);
    o.text("%% A # X %lld\n", 1);
    if (tmax) o.text("%% A + X %lld\n", tmax);
    index('A', ix_A);
    if (nR) o.text("# R %lld\n", nR);
    o.text("# D %lld\n", nalign);
    for (char t : {'T', 'X'}) {
      o.text(t == 'T' ? "# T %lld\n" : "# X %lld\n", nalign);
      if (tmax) o.text(t == 'T' ? "@ T %lld\n" : "@ X %lld\n", tmax);
      if (ttot) o.text(t == 'T' ? "+ T %lld\n" : "+ X %lld\n", ttot);
    }
  }
  o.text("^\n", 0);
  uint8_t off8[8];
  for (int b = 0; b < 8; b++) off8[b] = (uint8_t)((uint64_t)foot >> (8 * b));
  o.bytes(off8, 8);
  bool good = o.ok() && o.flush();
  good = !ferror(f) && good;
  if (fclose(f) != 0) good = false;
  return good ? PGA_OK : PGA_ERR_ARG;
}
