/* gdbdump [-s] <stem>
 *
 * Prints the contig table of a GDB as the reference reads it (Read_GDB,
 * lib/GDB.c:1171): one header line "ncontig maxctg seqtot f0 f1 f2 f3 seqpath"
 * and one "clen boff sbeg scaf" line per contig.  With -s it then prints
 * "nscaff hdrtot" and one "fctg ectg slen hoff <header>" line per scaffold.
 * Compiled only into oracle/_ref.  Test infrastructure.
 */
#include <stdio.h>
#include <stdlib.h>
#include "GDB.h"

int main(int argc, char *argv[])
{ GDB gdb;
  int i, scaffolds = 0;

  Prog_Name = "gdbdump";
  if (argc == 3 && argv[1][0] == '-' && argv[1][1] == 's')
    { scaffolds = 1;
      argv += 1;
      argc -= 1;
    }
  if (argc != 2)
    { fprintf(stderr, "usage: gdbdump [-s] <stem>\n");
      return 1;
    }
  if (Read_GDB(&gdb, argv[1]) < 0)
    { fprintf(stderr, "gdbdump: Read_GDB failed\n");
      return 1;
    }
  printf("%d %lld %lld %.9g %.9g %.9g %.9g %s\n", gdb.ncontig, (long long) gdb.maxctg,
         (long long) gdb.seqtot, gdb.freq[0], gdb.freq[1], gdb.freq[2], gdb.freq[3],
         gdb.seqpath ? gdb.seqpath : "-");
  for (i = 0; i < gdb.ncontig; i++)
    printf("%lld %lld %lld %d\n", (long long) gdb.contigs[i].clen, (long long) gdb.contigs[i].boff,
           (long long) gdb.contigs[i].sbeg, gdb.contigs[i].scaf);
  if (scaffolds)
    { printf("%d %lld\n", gdb.nscaff, (long long) gdb.hdrtot);
      for (i = 0; i < gdb.nscaff; i++)
        printf("%d %d %lld %lld %s\n", gdb.scaffolds[i].fctg, gdb.scaffolds[i].ectg,
               (long long) gdb.scaffolds[i].slen, (long long) gdb.scaffolds[i].hoff,
               gdb.headers + gdb.scaffolds[i].hoff);
    }
  Close_GDB(&gdb);
  return 0;
}
