/* assign_dump < input
 *
 * The reference's contig-pair -> rank assignment (contig_assignment_build,
 * src/contig_assignment.c) on given contig lengths.  Input (text): the
 * contig count N, the world size W, then N lengths.  Output: N lines of N
 * owners (-1 below the diagonal), then one line of W loads.  Compiled only
 * into oracle/_ref.  Test infrastructure.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "GDB.h"
#include "contig_assignment.h"

int main(void)
{ int               n, w, i, j;
  GDB               gdb;
  ContigAssignment  a;

  if (scanf("%d %d", &n, &w) != 2 || n <= 0)
    return 1;
  memset(&gdb, 0, sizeof(gdb));
  gdb.ncontig = n;
  gdb.contigs = calloc(n + 1, sizeof(GDB_CONTIG));
  for (i = 0; i < n; i++)
    { long long len;
      if (scanf("%lld", &len) != 1)
        return 1;
      gdb.contigs[i].clen = len;
    }
  if (contig_assignment_build(&gdb, w, &a) != 0)
    return 2;
  for (i = 0; i < n; i++)
    { for (j = 0; j < n; j++)
        printf(j ? " %d" : "%d", (int) a.rank_for_pair[(long long) i * n + j]);
      printf("\n");
    }
  for (i = 0; i < w; i++)
    printf(i ? " %lld" : "%lld", (long long) a.load_per_rank[i]);
  printf("\n");
  return 0;
}
