// The .1aln output of the alignment path: la_merge's file
// (src/fastga_pipeline.c:1616-1656) written as an ASCII ONE file.
//
// The reference writes the same records through ONElib in ONE's binary
// encoding (open_Aln_Write, lib/alncode.c:239-270).  ONE readers take either
// encoding, so the file here is ASCII: the header (file type "aln",
// provenance, references, the object counts readers use), the trace spacing
// line, the GDB skeleton (Write_Skeleton, lib/GDB.c:2059-2086) and one
// alignment per record in la_sort order (Write_Aln_Overlap / Write_Aln_Trace,
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

}  // namespace

extern "C" int pga_write_1aln(const char *path, const char *program, const char *version, const char *command,
                              const char *db_name, const char *cwd, int tspace, int nscaff,
                              const char *const *scaff_name, const int64_t *scaff_len, const int32_t *scaff_fctg,
                              const int64_t *contig_sbeg, const int64_t *contig_len, int64_t nalign,
                              const int32_t *recs9, const int64_t *trace_off, const uint8_t *trace) {
  if (!path || !program || !version || !command || !db_name || tspace <= 0 || nscaff < 0 || nalign < 0 ||
      (nscaff > 0 && (!scaff_name || !scaff_len || !scaff_fctg || !contig_sbeg || !contig_len)) ||
      (nalign > 0 && (!recs9 || !trace_off || !trace)))
    return PGA_ERR_ARG;
  for (int s = 0; s < nscaff; s++)
    if (!scaff_name[s] || strchr(scaff_name[s], '\n') || scaff_fctg[s + 1] < scaff_fctg[s]) return PGA_ERR_ARG;
  FILE *f = fopen(path, "w");
  if (!f) return PGA_ERR_ARG;

  // header
  char date[64];
  time_t now = time(nullptr);
  struct tm tmv;
  localtime_r(&now, &tmv);
  strftime(date, sizeof(date), "%F_%T", &tmv);
  int64_t tmax = 0, ttot = 0;
  for (int64_t i = 0; i < nalign; i++) {
    int64_t n = recs9[9 * i + 8] / 2;
    if (n > tmax) tmax = n;
    ttot += n;
  }
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
  fprintf(f, "\n.");
  // counts: objects and list sizes
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
