/* fa2gdb <in.fa> <out.1gdb>
 *
 * Builds a GDB (.1gdb + hidden .bps) from a FASTA file by calling the
 * reference's own Create_GDB / Write_GDB (lib/GDB.c:442, lib/GDB.c:1519);
 * FastGA's FAtoGDB is not part of the reference tree.  Compiled only into
 * oracle/_ref.  Test infrastructure.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "GDB.h"

int main(int argc, char *argv[])
{ GDB    gdb;
  FILE **units;
  char  *spath, *tpath;
  int    type;

  Prog_Name    = "fa2gdb";
  Command_Line = "fa2gdb";
  if (argc != 3)
    { fprintf(stderr, "usage: fa2gdb <in.fa> <out.1gdb>\n");
      return 1;
    }
  type  = Get_GDB_Paths(argv[1], argv[2], &spath, &tpath, 1);
  if (type < 0)
    { fprintf(stderr, "fa2gdb: cannot resolve %s -> %s\n", argv[1], argv[2]);
      return 1;
    }
  units = Create_GDB(&gdb, spath, type, 1, tpath, 0, NULL);
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
