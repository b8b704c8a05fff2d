/* split_dump < input
 *
 * The reference's stage-2 splitter (compute_destination_map, src/dsort.c)
 * on given global bucket counts.  Input (text): the world size W, then
 * NUM_BUCK counts.  Output: one line of ksplit[0..W], one line of
 * select[0..NUM_BUCK).  Compiled only into oracle/_ref.  Test
 * infrastructure.
 */
#include <stdio.h>
#include <stdlib.h>
#include "dsort.h"

int main(void)
{ int      w, i;
  int64_t  counts[NUM_BUCK];
  int     *ksplit, select[NUM_BUCK];

  if (scanf("%d", &w) != 1 || w <= 0)
    return 1;
  for (i = 0; i < NUM_BUCK; i++)
    { long long c;
      if (scanf("%lld", &c) != 1)
        return 1;
      counts[i] = c;
    }
  ksplit = calloc(w + 1, sizeof(int));
  compute_destination_map(counts, w, ksplit, select);
  for (i = 0; i <= w; i++)
    printf(i ? " %d" : "%d", ksplit[i]);
  printf("\n");
  for (i = 0; i < NUM_BUCK; i++)
    printf(i ? " %d" : "%d", select[i]);
  printf("\n");
  return 0;
}
