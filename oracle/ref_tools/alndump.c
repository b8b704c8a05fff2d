/* alndump [-s] <file.1aln>
 *
 * Prints the alignment record stream of a .1aln file, one alignment per line:
 *   aread abpos aepos bread bbpos bepos comp diffs ; T b-deltas ; X diffs
 * read with the reference's own reader (open_Aln_Read / Read_Aln_Overlap /
 * Read_Aln_Trace, lib/alncode.c:59-190).  The provenance and references
 * (which carry a timestamp and paths) are not printed; with -s the GDB
 * skeleton is, first, one line per S (scaffold name), G (gap) and C (contig
 * length) record.  Compiled only into oracle/_ref.  Test infrastructure.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "GDB.h"
#include "align.h"
#include "alncode.h"

int main(int argc, char *argv[])
{ OneFile *of;
  int64    novl, k;
  int      tspace, i;
  char    *db1, *db2, *cpath;
  uint8   *trace;
  Overlap  ovl;

  Prog_Name    = "alndump";
  Command_Line = "alndump";
  int skel = 0;
  if (argc == 3 && strcmp(argv[1], "-s") == 0)
    { skel = 1;
      argv += 1;
      argc -= 1;
    }
  if (argc != 2)
    { fprintf(stderr, "usage: alndump [-s] <file.1aln>\n");
      return 1;
    }
  of = open_Aln_Read(argv[1], 1, &novl, &tspace, &db1, &db2, &cpath);
  if (of == NULL)
    { fprintf(stderr, "alndump: cannot open %s\n", argv[1]);
      return 1;
    }
  if (skel)
    { while (of->lineType != 'A')          /* print the GDB skeleton */
        { if (of->lineType == 'S')
            printf("S %.*s\n", (int) oneLen(of), oneString(of));
          else if (of->lineType == 'G' || of->lineType == 'C')
            printf("%c %lld\n", of->lineType, (long long) oneInt(of, 0));
          if (!oneReadLine(of)) break;
        }
    }
  while (of->lineType == 'g')              /* skip the GDB skeleton */
    { Skip_Skeleton(of);
      if (of->lineType != 'A' && !oneReadLine(of)) break;
    }
  trace = malloc(1 << 24);
  printf("# tspace %d alignments %lld\n", tspace, (long long) novl);
  for (k = 0; k < novl; k++)
    { int tlen;
      if (of->lineType != 'A') break;
      Read_Aln_Overlap(of, &ovl);
      tlen = Read_Aln_Trace(of, trace, NULL);
      printf("%d %d %d %d %d %d %d %d ;", ovl.aread, ovl.path.abpos, ovl.path.aepos, ovl.bread,
             ovl.path.bbpos, ovl.path.bepos, COMP(ovl.flags) ? 1 : 0, ovl.path.diffs);
      for (i = 1; i < tlen; i += 2) printf(" %d", trace[i]);
      printf(" ;");
      for (i = 0; i < tlen; i += 2) printf(" %d", trace[i]);
      printf("\n");
    }
  free(trace);
  oneFileClose(of);
  return 0;
}
