/* onestat <file.1aln>
 *
 * Prints what a ONE reader learns about a .1aln file besides its records,
 * read with the reference's own ONElib (oneFileOpenRead with the aln schema
 * of lib/alncode.c:19-52):
 *   "binary" 0|1
 *   per line type with a count:   "# t count max total"       (oneStats)
 *   per object type, per line type it contains with a nonzero figure:
 *                                 "% t u maxCount maxTotal"   (oneStatsContains)
 *   for a binary file, every A, S and g object reached through the file's
 *   byte index (oneGoto), last object first:
 *                                 "@ t i fields..."
 * Compiled only into oracle/_ref.  Test infrastructure.
 */
#include <ctype.h>
#include <stdio.h>
#include <string.h>
#include "GDB.h"
#include "align.h"
#include "alncode.h"

int main(int argc, char *argv[])
{ OneSchema *vs;
  OneFile   *of;
  int        t, u;
  I64        n, mx, tot, i;

  if (argc != 2)
    { fprintf(stderr, "usage: onestat <file.1aln>\n");
      return 1;
    }
  vs = make_Aln_Schema();
  of = oneFileOpenRead(argv[1], vs, "aln", 1);
  if (of == NULL)
    { fprintf(stderr, "onestat: cannot open %s\n", argv[1]);
      return 1;
    }
  printf("binary %d\n", of->isBinary ? 1 : 0);
  for (t = 'A'; t <= 'z'; t++)
    { if (!isalpha(t) || of->info[t] == NULL)
        continue;
      if (!oneStats(of, (char) t, &n, &mx, &tot) || (n == 0 && mx == 0 && tot == 0))
        continue;
      printf("# %c %lld %lld %lld\n", t, (long long) n, (long long) mx, (long long) tot);
      if (!of->info[t]->isObject)
        continue;
      for (u = 'A'; u <= 'z'; u++)
        if (isalpha(u) && oneStatsContains(of, (char) t, (char) u, &n, &mx) && (n != 0 || mx != 0))
          printf("%% %c %c %lld %lld\n", t, u, (long long) n, (long long) mx);
    }
  if (of->isBinary)
    { const char *objs = "ASg";
      int k;
      for (k = 0; objs[k]; k++)
        { t = objs[k];
          oneStats(of, (char) t, &n, NULL, NULL);
          for (i = n; i >= 1; i--)
            { if (!oneGoto(of, (char) t, i) || oneReadLine(of) != t)
                { printf("@ %c %lld unreachable\n", t, (long long) i);
                  continue;
                }
              printf("@ %c %lld", t, (long long) i);
              if (t == 'A')
                { for (u = 0; u < 6; u++)
                    printf(" %lld", (long long) oneInt(of, u));
                }
              else if (t == 'S')
                printf(" %.*s", (int) oneLen(of), oneString(of));
              printf("\n");
            }
        }
    }
  oneFileClose(of);
  oneSchemaDestroy(vs);
  return 0;
}
