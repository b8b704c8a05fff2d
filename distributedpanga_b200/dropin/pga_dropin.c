/* The reference's stage entry points, with its exact signatures, over the
 * B200 library (include/pga_dropin.h says which and what each does).
 *
 * Linked into a build of the reference's driver in place of src/extract.c,
 * src/sort.c, src/kmer_adapter.c and src/fastga_pipeline.c, it keeps one
 * pga_ctx on the GPU for the whole run: the GDB's 2-bit image is uploaded
 * once, every stage's compute runs in libpga_b200.so, and the results come
 * back in the reference's byte formats and globals.  Compiled with the
 * reference's include paths (its lib/ and src/ and an mpi.h).
 */
#define _FILE_OFFSET_BITS 64
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include <sys/time.h>

#include "pga_dropin.h"
#include "pga_b200.h"

/* src/constants.h's KMER macro collides with the driver's KMER variable
 * (src/pga-mpi-merge.c:49-50 does the same). */
#undef KMER

/* The driver's globals these stages read and write (src/pga-mpi-merge.c:55-113). */
extern int NTHREADS, NUNITS, FREQ, KMER, CHAIN_BREAK, CHAIN_MIN, ALIGN_MIN, NCONTS, DBYTE;
extern double ALIGN_RATE;
extern int A_POSITION_BYTES, A_CONTIG_STRAND_BYTES;
extern int64 AMXPOS;
extern int8_t *RankForPair;
extern char *SORT_PATH, *ALGN_UNIQ;
extern IOBuffer *N_Units, *C_Units;
extern SeedUnit *N_SeedUnits, *C_SeedUnits;
extern uint8 *Recv_N_Data, *Recv_C_Data;
extern int64 Recv_N_Len, Recv_C_Len;

/* The globals the replaced files define. */
ExtractStats g_extract_stats;
PairSearchStats Pair_Search_Stats;
PairTaskHook Pair_Task_Hook = NULL;
SelfOrderHooks *Self_Order = NULL;

static pga_ctx *g_ctx = NULL;
static const GDB *g_loaded = NULL;  /* the GDB whose image the context holds */

static void die(const char *what, int rc) {
  fprintf(stderr, "%s: %s failed (%d): %s\n", Prog_Name ? Prog_Name : "pga_dropin", what, rc,
          g_ctx && pga_last_error(g_ctx) ? pga_last_error(g_ctx) : "");
  exit(1);
}

static void check(int rc, const char *what) {
  if (rc != PGA_OK) die(what, rc);
}

static double now_s(void) {
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static pga_ctx *context(void) {
  if (g_ctx == NULL) {
    const char *d = getenv("PGA_DEVICE");
    check(pga_ctx_create(d ? atoi(d) : 0, &g_ctx), "pga_ctx_create");
  }
  return g_ctx;
}

/* The GDB's 2-bit image (its .bps bytes: EXTERNAL reads the file, COMPRESSED
 * is already in memory), contig lengths and offsets, and base frequencies,
 * into the context -- once per GDB. */
static pga_ctx *context_for(GDB *gdb) {
  pga_ctx *ctx = context();
  if (g_loaded == gdb) return ctx;
  const int nc = gdb->ncontig;
  int64_t *clen = malloc(sizeof(int64_t) * (nc > 0 ? nc : 1));
  int64_t *boff = malloc(sizeof(int64_t) * (nc > 0 ? nc : 1));
  if (!clen || !boff) die("malloc", PGA_ERR_NOMEM);
  int64_t bytes = 0;
  for (int c = 0; c < nc; c++) {
    clen[c] = gdb->contigs[c].clen;
    boff[c] = gdb->contigs[c].boff;
    int64_t end = boff[c] + (clen[c] + 3) / 4;
    if (end > bytes) bytes = end;
  }
  uint8_t *image = NULL, *owned = NULL;
  if (gdb->seqstate == EXTERNAL) {
    FILE *f = (FILE *)gdb->seqs;
    if (f == NULL) die("GDB without sequence", PGA_ERR_ARG);
    owned = image = malloc(bytes > 0 ? bytes : 1);
    if (!image) die("malloc", PGA_ERR_NOMEM);
    if (bytes > 0 && (fseeko(f, 0, SEEK_SET) != 0 || fread(image, 1, bytes, f) != (size_t)bytes))
      die("reading the .bps file", PGA_ERR_ARG);
  } else if (gdb->seqstate == COMPRESSED) {
    image = (uint8_t *)gdb->seqs;
  } else {
    die("GDB sequence state (EXTERNAL or COMPRESSED needed)", PGA_ERR_ARG);
  }
  uint8_t one = 0;
  check(pga_gdb_load(ctx, bytes > 0 ? image : &one, bytes, nc, clen, boff), "pga_gdb_load");
  check(pga_gdb_set_freq(ctx, gdb->freq), "pga_gdb_set_freq");
  free(owned);
  free(clen);
  free(boff);
  g_loaded = gdb;
  return ctx;
}

/* ---- extraction (src/extract.c) ----------------------------------------- */

void extract_stats_reset(void) { memset(&g_extract_stats, 0, sizeof(g_extract_stats)); }

void record_buffer_init(RecordBuffer *b, RecordSizing sizing) {
  b->sizing = sizing;
  b->count = 0;
  b->capacity = 1 << 20;
  b->data = malloc((size_t)b->capacity * sizing.record_size + 1);  /* + the sentinel byte */
  if (!b->data) die("record_buffer_init", PGA_ERR_NOMEM);
}

void record_buffer_free(RecordBuffer *b) {
  free(b->data);
  b->data = NULL;
  b->count = b->capacity = 0;
}

void tuple_buffer_init(TupleBuffer *b) {
  b->data = NULL;
  b->count = b->capacity = 0;
}

void tuple_buffer_free(TupleBuffer *b) {
  free(b->data);
  b->data = NULL;
  b->count = b->capacity = 0;
}

void extract_to_records(GDB *gdb, int num_workers, int worker_id, RecordBuffer *buf) {
  pga_ctx *ctx = context_for(gdb);
  int posb, ctgb, rsize;
  check(pga_record_sizing(ctx, &posb, &ctgb, &rsize), "pga_record_sizing");
  if (rsize != buf->sizing.record_size || posb != buf->sizing.position_bytes ||
      ctgb != buf->sizing.contig_strand_bytes)
    die("record sizing differs from the buffer's", PGA_ERR_ARG);
  uint8_t *recs = NULL;
  int64_t n = 0;
  check(pga_extract_to_records(ctx, num_workers, worker_id, &recs, &n), "pga_extract_to_records");
  /* appended after what the buffer holds, with the sentinel byte after the last record */
  int64_t need = buf->count + n;
  if (need > buf->capacity || buf->data == NULL) {
    uint8_t *d = realloc(buf->data, (size_t)need * rsize + 1);
    if (!d) die("realloc", PGA_ERR_NOMEM);
    buf->data = d;
    buf->capacity = need;
  }
  memcpy(buf->data + buf->count * rsize, recs, (size_t)n * rsize);
  buf->count = need;
  buf->data[need * rsize] = 0;
  free(recs);
  /* the worker's contigs: split by cumulative bases as compute_work_split
   * (src/work_split.c:3-26) does */
  int *split = malloc(sizeof(int) * (num_workers + 1));
  if (!split) die("malloc", PGA_ERR_NOMEM);
  const int64_t total = gdb->seqtot;
  int64_t sofar = 0;
  for (int w = 0; w <= num_workers; w++) split[w] = w == num_workers ? gdb->ncontig : 0;
  int w = 1;
  int64_t next = total / num_workers;
  for (int c = 0; c < gdb->ncontig; c++) {
    sofar += gdb->contigs[c].clen;
    while (sofar >= next && w < num_workers) {
      split[w] = c + 1;
      w += 1;
      next = (total * w) / num_workers;
    }
  }
  for (int c = split[worker_id]; c < split[worker_id + 1]; c++) {
    g_extract_stats.contigs += 1;
    g_extract_stats.bases += gdb->contigs[c].clen;
  }
  free(split);
}

/* The same records as tuples (contig, position, strand, k-mer): decoded from
 * the record layout, appended to buf. */
void extract_to_tuples(GDB *gdb, int num_workers, int worker_id, TupleBuffer *buf) {
  pga_ctx *ctx = context_for(gdb);
  int posb, ctgb, rsize;
  check(pga_record_sizing(ctx, &posb, &ctgb, &rsize), "pga_record_sizing");
  RecordBuffer rb;
  rb.sizing.position_bytes = posb;
  rb.sizing.contig_strand_bytes = ctgb;
  rb.sizing.record_size = rsize;
  rb.data = NULL;
  rb.count = rb.capacity = 0;
  extract_to_records(gdb, num_workers, worker_id, &rb);
  const int64_t need = buf->count + rb.count;
  if (need > buf->capacity) {
    Tuple *d = realloc(buf->data, sizeof(Tuple) * (need > 0 ? need : 1));
    if (!d) die("realloc", PGA_ERR_NOMEM);
    buf->data = d;
    buf->capacity = need;
  }
  const int64_t smask = (int64_t)1 << (8 * ctgb - 1);
  for (int64_t i = 0; i < rb.count; i++) {
    const uint8_t *r = rb.data + i * rsize;
    int64_t pos = 0, cs = 0;
    memcpy(&pos, r + 12, posb);
    memcpy(&cs, r + 12 + posb, ctgb);
    Tuple *t = buf->data + buf->count + i;
    t->contig = (int)(cs & (smask - 1));
    t->strand = (cs & smask) ? 1 : 0;
    t->position = pos;
    memcpy(t->kmer, r + 1, 10);
  }
  buf->count = need;
  free(rb.data);
}

/* ---- sort + LCP (src/sort.c) ---------------------------------------------- */

void sort_records(RecordBuffer *buf) {
  check(pga_sort_records(context(), buf->data, buf->count, buf->sizing.position_bytes,
                         buf->sizing.contig_strand_bytes),
        "pga_sort_records");
}

void recalc_all_lcps(RecordBuffer *buf) {
  check(pga_recalc_lcps(context(), buf->data, buf->count, buf->sizing.position_bytes,
                        buf->sizing.contig_strand_bytes),
        "pga_recalc_lcps");
}

int simple_kmer_lcp_bases(const uint8_t *a, const uint8_t *b, int kbytes) {
  for (int i = 0; i < kbytes; i++) {
    const unsigned x = a[i] ^ b[i];
    if (x) return 4 * i + (x >= 0x40 ? 0 : x >= 0x10 ? 1 : x >= 0x04 ? 2 : 3);
  }
  return 4 * kbytes;
}

/* ---- k-mer table (src/kmer_adapter.c) ----------------------------------- */

/* first prefix p with cum[p] > i (the group entry i lies in), or num_prefixes */
static int group_of(const KmerStreamAdapter *t, int64 i) {
  int a = 0, b = t->num_prefixes;
  while (a < b) {
    const int m = a + (b - a) / 2;
    if (t->cumulative_count_by_prefix[m] > i) b = m;
    else a = m + 1;
  }
  return a;
}

int build_kmer_adapter(const RecordBuffer *buffer, KmerStreamAdapter *t, PayloadLayout *pl) {
  const int posb = buffer->sizing.position_bytes, ctgb = buffer->sizing.contig_strand_bytes;
  const int64 n = buffer->count;
  t->kmer_length_bases = 40;
  t->prefix_bytes = 3;
  t->kmer_bytes = 10;
  t->entry_kmer_suffix_bytes = 7;
  t->entry_bytes = 9 + posb + ctgb;
  t->prefix_plus_entry_bytes = 3 + t->entry_bytes;
  t->num_entries = n;
  t->num_prefixes = 1 << 24;
  t->entries = malloc((size_t)n * t->entry_bytes + 1);
  t->cumulative_count_by_prefix = malloc(sizeof(int64) * t->num_prefixes);
  if (!t->entries || !t->cumulative_count_by_prefix) {
    fprintf(stderr, "build_kmer_adapter: out of memory\n");
    free(t->entries);
    free(t->cumulative_count_by_prefix);
    return -1;
  }
  int64_t largest = 0;
  const int rc = pga_build_kmer_adapter(context(), buffer->data, n, posb, ctgb, t->entries,
                                        (int64_t *)t->cumulative_count_by_prefix, &largest);
  if (rc != PGA_OK) {
    fprintf(stderr, "build_kmer_adapter: pga_build_kmer_adapter failed (%d): %s\n", rc,
            pga_last_error(g_ctx) ? pga_last_error(g_ctx) : "");
    free(t->entries);
    free(t->cumulative_count_by_prefix);
    return -1;
  }
  t->entries_end = t->entries + n * t->entry_bytes;
  t->is_clone = 0;
  adapter_First_Kmer_Entry(t);
  pl->payload_bytes = posb + ctgb;
  pl->contig_strand_bytes = ctgb;
  pl->largest_prefix_group_num_entries = largest;
  return 0;
}

void free_kmer_adapter(KmerStreamAdapter *t, PayloadLayout *pl) {
  (void)pl;
  free(t->entries);
  free(t->cumulative_count_by_prefix);
  t->entries = NULL;
  t->cumulative_count_by_prefix = NULL;
}

void adapter_GoTo_Kmer_Index(KmerStreamAdapter *t, int64 i) {
  if (i >= t->num_entries) {
    t->current_entry = NULL;
    t->current_entry_index = t->num_entries;
    t->current_prefix = t->num_prefixes;
    return;
  }
  t->current_entry_index = i;
  t->current_entry = t->entries + i * t->entry_bytes;
  t->current_prefix = group_of(t, i);
}

void adapter_First_Kmer_Entry(KmerStreamAdapter *t) {
  adapter_GoTo_Kmer_Index(t, 0);
  if (t->num_entries == 0) {  /* an empty table still starts at its first entry slot */
    t->current_entry = t->entries;
    t->current_entry_index = 0;
  }
}

void adapter_Next_Kmer_Entry(KmerStreamAdapter *t) {
  const int64 i = t->current_entry_index + 1;
  if (i >= t->num_entries) {
    t->current_entry = NULL;
    t->current_entry_index = i;
    t->current_prefix = t->num_prefixes;
    return;
  }
  t->current_entry_index = i;
  t->current_entry += t->entry_bytes;
  while (t->current_prefix < t->num_prefixes && t->cumulative_count_by_prefix[t->current_prefix] <= i)
    t->current_prefix++;
}

KmerStreamAdapter *adapter_Clone_Kmer_Stream(KmerStreamAdapter *t) {
  KmerStreamAdapter *c = malloc(sizeof(KmerStreamAdapter));
  if (!c) die("malloc", PGA_ERR_NOMEM);
  *c = *t;
  c->is_clone = 1;
  return c;
}

void adapter_Free_Kmer_Stream(KmerStreamAdapter *t) {
  if (t->is_clone) free(t);
}

uint8 *adapter_Current_Entry(KmerStreamAdapter *t, uint8 *ent) {
  if (ent == NULL) {
    ent = malloc(t->prefix_plus_entry_bytes);
    if (!ent) die("malloc", PGA_ERR_NOMEM);
    if (t->current_entry == NULL) return ent;
  }
  ent[0] = (uint8)(t->current_prefix >> 16);
  ent[1] = (uint8)(t->current_prefix >> 8);
  ent[2] = (uint8)t->current_prefix;
  memcpy(ent + 3, t->current_entry, t->entry_bytes);
  return ent;
}

/* ---- adaptamer merge (src/fastga_pipeline.c:418-499) ---------------------- */

static void check_parameters(void) {
  if (KMER != 40 || CHAIN_BREAK != 2000 || CHAIN_MIN != 170 || ALIGN_MIN != 100 || ALIGN_RATE != 0.3 ||
      NTHREADS != 1) {
    fprintf(stderr, "%s: the B200 stages run KMER 40, CHAIN_BREAK 2000, CHAIN_MIN 170, ALIGN_MIN 100, "
                    "ALIGN_RATE 0.3 and NTHREADS 1 only\n", Prog_Name);
    exit(1);
  }
}

void self_adaptamer_merge(KmerStreamAdapter *t, PayloadLayout *pl, int64 g1len) {
  (void)g1len;
  check_parameters();
  const int ctgb = pl->contig_strand_bytes, posb = pl->payload_bytes - ctgb;
  const int sb = 1 + 2 * pl->payload_bytes;
  uint8_t *seeds[2] = {NULL, NULL};
  int64_t len[2] = {0, 0};
  int64_t *buck[2];
  buck[0] = calloc(NCONTS > 0 ? NCONTS : 1, sizeof(int64_t));
  buck[1] = calloc(NCONTS > 0 ? NCONTS : 1, sizeof(int64_t));
  if (!buck[0] || !buck[1]) die("calloc", PGA_ERR_NOMEM);
  check(pga_self_adaptamer_merge(context(), t->entries, (const int64_t *)t->cumulative_count_by_prefix,
                                 t->num_entries, posb, ctgb, FREQ, NCONTS, &seeds[0], &len[0], &seeds[1], &len[1],
                                 buck[0], buck[1]),
        "pga_self_adaptamer_merge");
  SeedUnit *units[2] = {N_SeedUnits, C_SeedUnits};
  IOBuffer *bk[2] = {N_Units, C_Units};
  for (int u = 0; u < 2; u++) {
    if (NUNITS <= 1) {
      seed_unit_ensure(&units[u][0], len[u]);
      memcpy(units[u][0].data + units[u][0].len, seeds[u], (size_t)len[u]);
      units[u][0].len += len[u];
    } else {
      /* each seed to the unit of the rank owning its contig pair */
      const int64 cmask = ((int64)1 << (8 * ctgb - 1)) - 1;
      for (int64_t s = 0; s < len[u]; s += sb) {
        const uint8_t *x = seeds[u] + s;
        int64 a = 0, b = 0;
        memcpy(&a, x + 1 + posb, ctgb);
        memcpy(&b, x + 1 + pl->payload_bytes + posb, ctgb);
        const int r = RankForPair[(a & cmask) * NCONTS + (b & cmask)];
        seed_unit_ensure(&units[u][r], sb);
        memcpy(units[u][r].data + units[u][r].len, x, sb);
        units[u][r].len += sb;
      }
    }
    for (int c = 0; c < NCONTS; c++) bk[u][0].buck[c] += buck[u][c];
    free(seeds[u]);
    free(buck[u]);
  }
}

/* ---- diagonal sort, chaining, alignment, .1aln (src/fastga_pipeline.c:1686-1842) */

void pair_sort_search(GDB *gdb1, GDB *gdb2) {
  (void)gdb2;  /* self mode: gdb2 is gdb1 */
  check_parameters();
  pga_ctx *ctx = context_for(gdb1);
  memset(&Pair_Search_Stats, 0, sizeof(Pair_Search_Stats));
  const int sb = 1 + 2 * (A_POSITION_BYTES + A_CONTIG_STRAND_BYTES);
  double t0 = now_s();
  check(pga_seeds_load(ctx, 0, Recv_N_Data, Recv_N_Len), "pga_seeds_load");
  check(pga_seeds_load(ctx, 1, Recv_C_Data, Recv_C_Len), "pga_seeds_load");
  Pair_Search_Stats.nels[0] = Recv_N_Len / sb;
  Pair_Search_Stats.nels[1] = Recv_C_Len / sb;
  free(Recv_N_Data);
  free(Recv_C_Data);
  Recv_N_Data = Recv_C_Data = NULL;
  Recv_N_Len = Recv_C_Len = 0;
  Pair_Search_Stats.reimport_s[0] = now_s() - t0;
  t0 = now_s();
  int64_t nalign = 0;
  check(pga_align(ctx, &nalign), "pga_align");
  Pair_Search_Stats.search_s[0] = now_s() - t0;
  /* la_merge's file: ONE "aln" in the binary encoding open_Aln_Write asks
   * for, its provenance and references, the skeleton of gdb1
   * (Write_Skeleton, lib/GDB.c:2059), then the alignments in la_sort order */
  t0 = now_s();
  const int ns = gdb1->nscaff;
  const char **names = malloc(sizeof(char *) * (ns > 0 ? ns : 1));
  int64_t *slen = malloc(sizeof(int64_t) * (ns > 0 ? ns : 1));
  int32_t *fctg = malloc(sizeof(int32_t) * (ns + 1));
  int64_t *sbeg = malloc(sizeof(int64_t) * (gdb1->ncontig > 0 ? gdb1->ncontig : 1));
  if (!names || !slen || !fctg || !sbeg) die("malloc", PGA_ERR_NOMEM);
  for (int s = 0; s < ns; s++) {
    names[s] = gdb1->headers + gdb1->scaffolds[s].hoff;
    slen[s] = gdb1->scaffolds[s].slen;
    fctg[s] = gdb1->scaffolds[s].fctg;
  }
  fctg[ns] = ns > 0 ? gdb1->scaffolds[ns - 1].ectg : 0;
  for (int c = 0; c < gdb1->ncontig; c++) sbeg[c] = gdb1->contigs[c].sbeg;
  const size_t plen = strlen(SORT_PATH) + strlen(ALGN_UNIQ) + 8;
  char *path = malloc(plen);
  char *cwd = getcwd(NULL, 0);
  if (!path) die("malloc", PGA_ERR_NOMEM);
  snprintf(path, plen, "%s/%s.1aln", SORT_PATH, ALGN_UNIQ);
  check(pga_align_write_1aln_binary(ctx, path, "pga-merge", "0.1", "pga-merge", path, cwd, ns, names, slen, fctg,
                                    sbeg),
        "pga_align_write_1aln_binary");
  Pair_Search_Stats.la_merge_s = now_s() - t0;
  free(cwd);
  free(path);
  free(names);
  free(slen);
  free(fctg);
  free(sbeg);
}
