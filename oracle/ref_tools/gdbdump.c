/* gdbdump <stem>
 *
 * Prints the contig table of a GDB as the reference reads it (Read_GDB,
 * lib/GDB.c:1171): one header line "ncontig maxctg seqtot f0 f1 f2 f3 seqpath"
 * and one "clen boff sbeg scaf" line per contig.  Compiled only into
 * oracle/_ref.  Test infrastructure.
 */
#include <stdio.h>
#include <stdlib.h>
#include "GDB.h"

int main(int argc, char *argv[])
{ GDB gdb;
  int i;

  Prog_Name = "gdbdump";
  if (argc != 2)
    { fprintf(stderr, "usage: gdbdump <stem>\n");
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
  Close_GDB(&gdb);
  return 0;
}
