/* la_batch <stem> <requests>
 *
 * Runs the reference's own Local_Alignment (lib/align.c:1423) on a list of
 * requests against the contigs of a GDB, set up as align_contigs sets it up
 * (src/fastga_pipeline.c:1086-1101, 720-730): NUMERIC contig buffers
 * (Get_Contig), A complemented in place for a reverse-complement request
 * (Complement_Seq, ACOMP_FLAG), New_Align_Spec(0.7, 100, freq, 0).
 * Each request line is "a b comp low hgh anti lbord hbord"; each output line
 * is "abpos aepos bbpos bepos diffs tlen ; t0 t1 ..." with the tlen uint16
 * trace values Local_Alignment leaves in its work data.  Compiled only into
 * oracle/_ref.  Test infrastructure.
 */
#include <stdio.h>
#include <stdlib.h>
#include "GDB.h"
#include "align.h"

int main(int argc, char *argv[])
{ GDB        gdb;
  FILE      *f;
  char      *aseq, *bseq;
  Work_Data *work;
  Align_Spec *spec;
  Alignment  align;
  Path       path;
  int        a, b, comp, low, hgh, anti, lbord, hbord, i;

  Prog_Name = "la_batch";
  if (argc != 3)
    { fprintf(stderr, "usage: la_batch <stem> <requests>\n");
      return 1;
    }
  if (Read_GDB(&gdb, argv[1]) < 0)
    { fprintf(stderr, "la_batch: Read_GDB failed\n");
      return 1;
    }
  f = fopen(argv[2], "r");
  if (f == NULL)
    { fprintf(stderr, "la_batch: cannot open %s\n", argv[2]);
      return 1;
    }
  aseq = New_Contig_Buffer(&gdb);
  bseq = New_Contig_Buffer(&gdb);
  work = New_Work_Data();
  spec = New_Align_Spec(1. - .3, 100, gdb.freq, 0);
  if (aseq == NULL || bseq == NULL || work == NULL || spec == NULL) return 1;
  align.path = &path;
  align.aseq = aseq;
  align.bseq = bseq;
  while (fscanf(f, "%d %d %d %d %d %d %d %d", &a, &b, &comp, &low, &hgh, &anti, &lbord, &hbord) == 8)
    { if (Get_Contig(&gdb, a, NUMERIC, aseq) == NULL) return 1;
      if (Get_Contig(&gdb, b, NUMERIC, bseq) == NULL) return 1;
      align.alen  = gdb.contigs[a].clen;
      align.blen  = gdb.contigs[b].clen;
      align.flags = comp ? ACOMP_FLAG : 0;
      if (comp) Complement_Seq(aseq, align.alen);
      if (Local_Alignment(&align, work, spec, low, hgh, anti, lbord, hbord))
        { fprintf(stderr, "la_batch: Local_Alignment failed\n");
          return 1;
        }
      printf("%d %d %d %d %d %d ;", path.abpos, path.aepos, path.bbpos, path.bepos, path.diffs, path.tlen);
      for (i = 0; i < path.tlen; i++)
        printf(" %d", ((uint16 *) path.trace)[i]);
      printf("\n");
    }
  fclose(f);
  Close_GDB(&gdb);
  return 0;
}
