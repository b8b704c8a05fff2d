/* Dump hooks for the reference driver built as the oracle (oracle/_ref).
 *
 * src/pga-mpi-merge.c is compiled unchanged except that its calls to
 * build_kmer_adapter (src/pga-mpi-merge.c:384) and pair_sort_search
 * (src/pga-mpi-merge.c:588) are renamed to the two functions below, which
 * write the stage's input to $ORACLE_DUMP_DIR and then call the real
 * function.  Files written:
 *
 *   index.bin  int32 rsize, posb, ctgb; int64 count; then count records of
 *              rsize bytes exactly as run_stage2 left them (sorted by k-mer,
 *              byte 0 = LCP in bases)
 *   seeds.bin  int32 seed_bytes, ncontig; int64 nlen, clen; N seed bytes;
 *              C seed bytes; int64 nbuck[ncontig]; int64 cbuck[ncontig]
 *   diag_N.bin, diag_C.bin
 *              int32 swide, ncontig; int64 nels; the sort array after
 *              rmsd_sort; int64 panel[ncontig] (bytes per A-contig panel).
 *              rmsd_sort is reached through src/fastga_pipeline.c:1822, whose
 *              call is renamed to oracle_hook_rmsd_sort; N is sorted first.
 *
 * Test infrastructure.
 */
#include <stdio.h>
#include <stdlib.h>
#include <stdint.h>
#include <string.h>
#include "GDB.h"
#include "extract.h"
#include "kmer_adapter.h"
#include "fastga_pipeline.h"

extern uint8    *Recv_N_Data;
extern uint8    *Recv_C_Data;
extern int64     Recv_N_Len;
extern int64     Recv_C_Len;
extern IOBuffer *N_Units;
extern IOBuffer *C_Units;
extern int       NCONTS;
extern int       A_PAYLOAD_BYTES, B_PAYLOAD_BYTES;

static FILE *dump_open(const char *name)
{ const char *dir = getenv("ORACLE_DUMP_DIR");
  char path[4096];
  FILE *f;
  if (dir == NULL || dir[0] == '\0') return NULL;
  snprintf(path, sizeof(path), "%s/%s", dir, name);
  f = fopen(path, "wb");
  if (f == NULL) { fprintf(stderr, "ref_hooks: cannot open %s\n", path); exit(1); }
  return f;
}

int oracle_hook_build_kmer_adapter(const RecordBuffer *buffer, KmerStreamAdapter *t, PayloadLayout *p)
{ FILE *f = dump_open("index.bin");
  if (f != NULL)
    { int32_t hdr[3] = { buffer->sizing.record_size, buffer->sizing.position_bytes,
                         buffer->sizing.contig_strand_bytes };
      int64_t n = buffer->count;
      fwrite(hdr, sizeof(hdr), 1, f);
      fwrite(&n, sizeof(n), 1, f);
      if (n > 0) fwrite(buffer->data, (size_t) buffer->sizing.record_size, (size_t) n, f);
      fclose(f);
    }
  return build_kmer_adapter(buffer, t, p);
}

void oracle_hook_pair_sort_search(GDB *g1, GDB *g2)
{ FILE *f = dump_open("seeds.bin");
  if (f != NULL)
    { int32_t hdr[2] = { 1 + A_PAYLOAD_BYTES + B_PAYLOAD_BYTES, NCONTS };
      int64_t lens[2] = { Recv_N_Len, Recv_C_Len };
      fwrite(hdr, sizeof(hdr), 1, f);
      fwrite(lens, sizeof(lens), 1, f);
      if (Recv_N_Len > 0) fwrite(Recv_N_Data, 1, (size_t) Recv_N_Len, f);
      if (Recv_C_Len > 0) fwrite(Recv_C_Data, 1, (size_t) Recv_C_Len, f);
      fwrite(N_Units[0].buck, sizeof(int64), (size_t) NCONTS, f);
      fwrite(C_Units[0].buck, sizeof(int64), (size_t) NCONTS, f);
      fclose(f);
    }
  pair_sort_search(g1, g2);
}

extern int rmsd_sort(uint8 *array, int64 nelem, int rsize, int ksize,
                     int nparts, int64 *part, int nthreads, void *parms);

int oracle_hook_rmsd_sort(uint8 *array, int64 nelem, int rsize, int ksize,
                          int nparts, int64 *part, int nthreads, void *parms)
{ static int calls = 0;
  int64_t *panel = malloc(sizeof(int64_t) * (size_t) (nparts > 0 ? nparts : 1));
  int r;
  FILE *f;
  if (nparts > 0) memcpy(panel, part, sizeof(int64_t) * (size_t) nparts);
  r = rmsd_sort(array, nelem, rsize, ksize, nparts, part, nthreads, parms);
  f = dump_open(calls == 0 ? "diag_N.bin" : "diag_C.bin");
  calls += 1;
  if (f != NULL)
    { int32_t hdr[2] = { rsize, nparts };
      int64_t n = nelem;
      fwrite(hdr, sizeof(hdr), 1, f);
      fwrite(&n, sizeof(n), 1, f);
      if (n > 0) fwrite(array, (size_t) rsize, (size_t) n, f);
      fwrite(panel, sizeof(int64_t), (size_t) nparts, f);
      fclose(f);
    }
  free(panel);
  return r;
}
