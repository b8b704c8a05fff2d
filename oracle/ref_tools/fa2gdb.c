/* fa2gdb <in.fa> <out.1gdb> [nthr]
 *
 * Builds a GDB (.1gdb + hidden .bps) from a FASTA file by calling the
 * reference's own Create_GDB / Write_GDB (lib/GDB.c:442, lib/GDB.c:1519);
 * FastGA's FAtoGDB is not part of the reference tree.  nthr (default 0, as
 * the reference's own call at lib/GDB.c:1662) is Create_GDB's gap threshold.
 * Compiled only into oracle/_ref.  Test infrastructure.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "GDB.h"

int main(int argc, char *argv[])
{ GDB    gdb;
  FILE **units;
  char  *spath, *tpath;
  int    type, nthr;

  Prog_Name    = "fa2gdb";
  Command_Line = "fa2gdb";
  if (argc != 3 && argc != 4)
    { fprintf(stderr, "usage: fa2gdb <in.fa> <out.1gdb> [nthr]\n");
      return 1;
    }
  nthr = argc == 4 ? atoi(argv[3]) : 0;
  type  = Get_GDB_Paths(argv[1], argv[2], &spath, &tpath, 1);
  if (type < 0)
    { fprintf(stderr, "fa2gdb: cannot resolve %s -> %s\n", argv[1], argv[2]);
      return 1;
    }
  units = Create_GDB(&gdb, spath, type, 1, tpath, nthr, NULL);
  if (units == NULL)
    { fprintf(stderr, "fa2gdb: Create_GDB failed\n");
      return 1;
    }
  if (Write_GDB(&gdb, tpath))
    { fprintf(stderr, "fa2gdb: Write_GDB failed\n");
      return 1;
    }
  Close_GDB(&gdb);
  return 0;
}
