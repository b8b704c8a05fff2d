/* alnwrite <in.1aln> <ref_out.1aln> <pga_out.1aln>
 *
 * A C caller of libpga_b200 that holds its alignments in the reference's
 * own types.  It reads in.1aln with the reference's reader (open_Aln_Read,
 * Read_Skeleton, Read_Aln_Overlap / Read_Aln_Trace, lib/alncode.c and
 * lib/GDB.c) into Overlap records, their trace bytes and a GDB skeleton,
 * then writes them twice:
 *   ref_out.1aln  through the reference's writer, as la_merge does
 *                 (open_Aln_Write, Write_Skeleton, Write_Aln_Overlap,
 *                 Write_Aln_Trace; src/fastga_pipeline.c:1616-1656);
 *   pga_out.1aln  through pga_write_1aln_binary (include/pga_b200.h), its
 *                 arguments taken from those same structures.
 * Compiled only into oracle/_ref.  Test infrastructure.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "GDB.h"
#include "align.h"
#include "alncode.h"
#include "pga_b200.h"

int main(int argc, char *argv[])
{ OneFile *in, *out;
  int64    novl, k, nread, tbytes, tcap;
  int      tspace, have_skel, s, c, tlen;
  char    *db1, *db2, *cpath;
  GDB      gdb;
  Overlap *ovl;
  uint8   *tbuf, *trace;
  int64   *toff, *t64, tlmax;
  int32_t *recs9;

  Prog_Name    = "alnwrite";
  Command_Line = "alnwrite";
  if (argc != 4)
    { fprintf(stderr, "usage: alnwrite <in.1aln> <ref_out.1aln> <pga_out.1aln>\n");
      return 1;
    }
  db1 = db2 = cpath = NULL;
  in = open_Aln_Read(argv[1], 1, &novl, &tspace, &db1, &db2, &cpath);
  if (in == NULL)
    { fprintf(stderr, "alnwrite: cannot open %s\n", argv[1]);
      return 1;
    }
  have_skel = 0;
  memset(&gdb, 0, sizeof(gdb));
  if (in->lineType == 'g')
    { if (Read_Skeleton(in, "skeleton.fa", &gdb))
        { fprintf(stderr, "alnwrite: cannot read the skeleton\n");
          return 1;
        }
      have_skel = 1;
    }

  /* the records in the reference's Overlap, their traces back to back
     (a trace holds 2 bytes per T value; the file's largest T list sizes it) */
  { I64 tmax = 0;
    oneStats(in, 'T', NULL, &tmax, NULL);
    tlmax = 2 * (tmax > 0 ? tmax : 1);
  }
  ovl   = malloc(sizeof(Overlap) * (novl > 0 ? novl : 1));
  toff  = malloc(sizeof(int64) * (novl + 1));
  tbuf  = malloc(tlmax);
  tcap  = 1 << 20;
  trace = malloc(tcap);
  tbytes = 0;
  nread  = 0;
  toff[0] = 0;
  for (k = 0; k < novl && in->lineType == 'A'; k++)
    { Read_Aln_Overlap(in, &ovl[k]);
      tlen = Read_Aln_Trace(in, tbuf, NULL);
      if (tbytes + tlen > tcap)
        { while (tbytes + tlen > tcap)
            tcap *= 2;
          trace = realloc(trace, tcap);
        }
      memcpy(trace + tbytes, tbuf, tlen);
      ovl[k].path.tlen = tlen;
      tbytes += tlen;
      toff[k + 1] = tbytes;
      nread += 1;
    }
  oneFileClose(in);
  if (nread != novl)
    { fprintf(stderr, "alnwrite: %lld of %lld alignments read\n", (long long) nread, (long long) novl);
      return 1;
    }

  /* the reference's writer */
  out = open_Aln_Write(argv[2], 1, "alnwrite", "1", "alnwrite", tspace, db1, db2, cpath);
  if (out == NULL)
    return 1;
  if (have_skel)
    Write_Skeleton(out, &gdb);
  t64 = malloc(sizeof(int64) * tlmax);
  for (k = 0; k < novl; k++)
    { Write_Aln_Overlap(out, &ovl[k]);
      Write_Aln_Trace(out, trace + toff[k], ovl[k].path.tlen, t64, 0);
    }
  oneFileClose(out);

  /* libpga_b200 from the same structures */
  { int          ns = have_skel ? gdb.nscaff : 0;
    const char **names = malloc(sizeof(char *) * (ns > 0 ? ns : 1));
    int64_t     *slen  = malloc(sizeof(int64_t) * (ns > 0 ? ns : 1));
    int32_t     *fctg  = malloc(sizeof(int32_t) * (ns + 1));
    int64_t     *sbeg  = malloc(sizeof(int64_t) * (gdb.ncontig > 0 ? gdb.ncontig : 1));
    int64_t     *clen  = malloc(sizeof(int64_t) * (gdb.ncontig > 0 ? gdb.ncontig : 1));
    int          rc;

    for (s = 0; s < ns; s++)
      { names[s] = gdb.headers + gdb.scaffolds[s].hoff;
        slen[s]  = gdb.scaffolds[s].slen;
        fctg[s]  = gdb.scaffolds[s].fctg;
      }
    fctg[ns] = ns > 0 ? gdb.scaffolds[ns - 1].ectg : 0;
    for (c = 0; c < (have_skel ? gdb.ncontig : 0); c++)
      { sbeg[c] = gdb.contigs[c].sbeg;
        clen[c] = gdb.contigs[c].clen;
      }
    recs9 = malloc(sizeof(int32_t) * 9 * (novl > 0 ? novl : 1));
    for (k = 0; k < novl; k++)
      { int32_t *r = recs9 + 9 * k;
        r[0] = ovl[k].aread;
        r[1] = ovl[k].path.abpos;
        r[2] = ovl[k].path.aepos;
        r[3] = ovl[k].bread;
        r[4] = ovl[k].path.bbpos;
        r[5] = ovl[k].path.bepos;
        r[6] = COMP(ovl[k].flags) ? 1 : 0;
        r[7] = ovl[k].path.diffs;
        r[8] = ovl[k].path.tlen;
      }
    rc = pga_write_1aln_binary(argv[3], "alnwrite", "1", "alnwrite", db1, (cpath && *cpath) ? cpath : NULL,
                               tspace, ns, names, slen, fctg, sbeg, clen, novl, recs9, (const int64_t *) toff,
                               trace);
    if (rc != PGA_OK)
      { fprintf(stderr, "alnwrite: pga_write_1aln_binary returned %d\n", rc);
        return 1;
      }
  }
  printf("%lld alignments, %d scaffolds\n", (long long) novl, have_skel ? gdb.nscaff : 0);
  return 0;
}
