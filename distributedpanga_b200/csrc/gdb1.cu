// A GDB on disk: the .1gdb skeleton (ONE file type "gdb") and the hidden
// .bps sequence file beside it, as Write_GDB (lib/GDB.c:1519-1608) leaves
// them after Create_GDB.
//
// The .1gdb is written in ONE's ASCII encoding (the reference writes the
// same lines in the binary one; ONE readers take either): the header
// (provenance, the source FASTA as reference, the schema, the object
// counts Read_GDB sizes its tables from, lib/GDB.c:1251-1254), the base
// frequencies, then per scaffold its name and its gaps and contigs in order:
//
//   f A C G T       base frequencies
//   S name          one scaffold
//   G length        a gap
//   C length        a contig
//
// The .bps is <dir>/.<root>.bps for tpath <dir>/<root>.1gdb (or .gdb): the
// 2-bit image, each contig from a fresh byte.  Host code only.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <string>
#include "../../include/pga_b200.h"

namespace {

constexpr int ONE_MAJOR = 2, ONE_MINOR = 1;

// The "gdb" file type's line definitions (lib/GDB.c:37-47).
const char *const GDB_SCHEMA[] = {
    "D f 4 4 REAL 4 REAL 4 REAL 4 REAL",
    "D u 0",
    "O S 1 6 STRING",
    "D G 1 3 INT",
    "D C 1 3 INT",
    "D M 1 8 INT_LIST",
};

void put_string(FILE *f, const char *s, size_t n) {
  fprintf(f, " %zu ", n);
  fwrite(s, 1, n, f);
}

// <dir>/.<root>.bps for <dir>/<root>.1gdb or <dir>/<root>.gdb (lib/GDB.c:1533-1546).
bool bps_path(const char *tpath, std::string *out) {
  std::string t(tpath);
  size_t slash = t.rfind('/');
  std::string dir = slash == std::string::npos ? "." : t.substr(0, slash);
  std::string base = slash == std::string::npos ? t : t.substr(slash + 1);
  const char *ext[2] = {".1gdb", ".gdb"};
  for (const char *e : ext) {
    size_t k = strlen(e);
    if (base.size() > k && base.compare(base.size() - k, k, e) == 0) {
      *out = dir + "/." + base.substr(0, base.size() - k) + ".bps";
      return true;
    }
  }
  return false;
}

}  // namespace

extern "C" int pga_write_1gdb(const char *tpath, const char *program, const char *version, const char *command,
                              const char *srcpath, const float *freq4, int nscaff, const int64_t *scaffolds4,
                              const char *headers, int64_t hdrtot, int ncontig, const int64_t *contigs4,
                              const uint8_t *bps, int64_t bps_bytes) {
  if (!tpath || !program || !version || !command || !srcpath || !freq4 || nscaff < 1 || ncontig < 1 ||
      !scaffolds4 || !headers || hdrtot < nscaff || !contigs4 || bps_bytes < 0 || (bps_bytes > 0 && !bps))
    return PGA_ERR_ARG;
  for (int s = 0; s < nscaff; s++) {
    const int64_t *r = scaffolds4 + 4 * s;
    if (r[0] < 0 || r[1] < r[0] || r[1] > ncontig || r[3] < 0 || r[3] >= hdrtot) return PGA_ERR_ARG;
    if (!memchr(headers + r[3], 0, (size_t)(hdrtot - r[3]))) return PGA_ERR_ARG;
  }
  std::string bpath;
  if (!bps_path(tpath, &bpath)) return PGA_ERR_ARG;

  FILE *b = fopen(bpath.c_str(), "wb");
  if (!b) return PGA_ERR_ARG;
  bool bad = bps_bytes > 0 && fwrite(bps, 1, (size_t)bps_bytes, b) != (size_t)bps_bytes;
  if (fclose(b) != 0) bad = true;
  if (bad) return PGA_ERR_ARG;

  FILE *f = fopen(tpath, "w");
  if (!f) return PGA_ERR_ARG;
  char date[64];
  time_t now = time(nullptr);
  struct tm tmv;
  localtime_r(&now, &tmv);
  strftime(date, sizeof(date), "%F_%T", &tmv);

  int64_t maxname = 0, ngap = 0;
  for (int s = 0; s < nscaff; s++) {
    const int64_t *r = scaffolds4 + 4 * s;
    int64_t len = (int64_t)strlen(headers + r[3]);
    if (len > maxname) maxname = len;
    int64_t spos = 0;
    for (int64_t c = r[0]; c < r[1]; c++) {
      if (contigs4[4 * c + 2] > spos) ngap++;
      spos = contigs4[4 * c + 2] + contigs4[4 * c + 0];
    }
    if (r[2] > spos) ngap++;
  }

  fprintf(f, "1 3 gdb %d %d", ONE_MAJOR, ONE_MINOR);
  fprintf(f, "\n! 4");
  put_string(f, program, strlen(program));
  put_string(f, version, strlen(version));
  put_string(f, command, strlen(command));
  put_string(f, date, strlen(date));
  fprintf(f, "\n.");
  fprintf(f, "\n<");
  put_string(f, srcpath, strlen(srcpath));
  fprintf(f, " 1");
  fprintf(f, "\n.");
  for (const char *d : GDB_SCHEMA) fprintf(f, "\n~ %s", d);
  fprintf(f, "\n.");
  fprintf(f, "\n# f 1");
  fprintf(f, "\n# S %d\n@ S %lld\n+ S %lld", nscaff, (long long)maxname, (long long)(hdrtot - nscaff));
  fprintf(f, "\n# G %lld", (long long)ngap);
  fprintf(f, "\n# C %d", ncontig);
  fprintf(f, "\n.");

  // Write_GDB's body (lib/GDB.c:1578-1604)
  fprintf(f, "\nf %.17g %.17g %.17g %.17g", (double)freq4[0], (double)freq4[1], (double)freq4[2],
          (double)freq4[3]);
  for (int s = 0; s < nscaff; s++) {
    const int64_t *r = scaffolds4 + 4 * s;
    const char *name = headers + r[3];
    fprintf(f, "\nS");
    put_string(f, name, strlen(name));
    int64_t spos = 0;
    for (int64_t c = r[0]; c < r[1]; c++) {
      const int64_t *q = contigs4 + 4 * c;
      if (q[2] > spos) fprintf(f, "\nG %lld", (long long)(q[2] - spos));
      fprintf(f, "\nC %lld", (long long)q[0]);
      spos = q[2] + q[0];
    }
    if (r[2] > spos) fprintf(f, "\nG %lld", (long long)(r[2] - spos));
  }
  fprintf(f, "\n");
  bad = ferror(f) != 0;
  if (fclose(f) != 0) bad = true;
  return bad ? PGA_ERR_ARG : PGA_OK;
}
