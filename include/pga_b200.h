/* pga_b200 -- B200 (sm_100a) implementation of DistributedPanGA's FastGA
 * alignment path, behind a plain C ABI.
 *
 * Two kinds of entry points:
 *
 *  1. Drop-in stages.  Each takes and returns host buffers in the reference's
 *     own byte formats and replaces one reference function at world size 1
 *     (the function is named beside it).  Buffers the reference allocates
 *     with malloc are allocated here with malloc too; free them with free().
 *
 *  2. The resident pipeline.  pga_gdb_load puts a GDB's 2-bit sequence and
 *     contig table in HBM; pga_index_build, pga_merge and pga_diag_sort then
 *     run extraction -> index sort -> LCPs -> k-mer table -> adaptamer merge ->
 *     seed reimport -> diagonal sort without leaving the device; the
 *     pga_*_copy functions read any stage's result back in the reference's
 *     format.
 *
 * Every function returns PGA_OK or an error code; pga_last_error() gives
 * the message.  A context is not thread-safe; use one per host thread.
 * Limits: contigs < 32768 (contig|strand fits 2 bytes), contig length
 * < 2^31, fewer than 2^32 - 1 k-mer records and seeds per unit.
 */
#ifndef PGA_B200_H
#define PGA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PGA_OK            0
#define PGA_ERR_CUDA      1   /* a CUDA call failed (message has the CUDA error) */
#define PGA_ERR_ARG       2   /* bad argument or call order */
#define PGA_ERR_NOMEM     3   /* device or host allocation failed */
#define PGA_ERR_LIMIT     4   /* input beyond the limits above */

typedef struct pga_ctx pga_ctx;
typedef struct pga_target pga_target;

/* ---- context ------------------------------------------------------------ */

int         pga_ctx_create(int device, pga_ctx **out);
void        pga_ctx_destroy(pga_ctx *ctx);
const char *pga_last_error(const pga_ctx *ctx);
/* Run the context's work on an existing cudaStream_t (NULL: the context's
 * own stream).  Lets a caller bracket the kernels with its own events. */
int         pga_ctx_set_stream(pga_ctx *ctx, void *stream);
int         pga_ctx_synchronize(pga_ctx *ctx);
/* Number of kernels this context has launched so far. */
int64_t     pga_kernel_launches(const pga_ctx *ctx);
/* Per-stage device times (ms) of the last pipeline calls when timing is on:
 * [0] extract+histogram [1] prefix scan [2] extract+scatter [3] bucket sort
 * [4] LCP [5] k-mer entries+prefix table [6] merge [7] diagonal sort of the
 * N unit [8] alignment (pga_align, host steps included) [9] diagonal sort of
 * the C unit. */
int         pga_ctx_enable_timing(pga_ctx *ctx, int on);
int         pga_stage_times(const pga_ctx *ctx, float *ms10);
/* Device memory.  A context keeps the memory it frees (an arena of slabs
 * from cudaMalloc) and hands it out again, so a repeated pipeline pass makes
 * no driver allocation calls; the memory goes back to the driver when the
 * context is destroyed, or when a request does not fit and slabs with
 * nothing live in them are returned to make room.  ms11: host time (ms)
 * inside cudaMalloc / cudaFree since timing was last enabled, charged to the
 * stage that asked ([0..9] as above, [10] outside every stage); counts4
 * (may be NULL): driver calls, bytes held, bytes held but free, times the
 * alignment buffers were freed to make room. */
int         pga_alloc_times(const pga_ctx *ctx, double *ms11, int64_t *counts4);

/* ---- GDB ------------------------------------------------------------------ */

/* Replaces reading the GDB's sequence for extraction (Read_GDB
 * lib/GDB.c:1171 + Get_Contig_Piece lib/GDB.c:1831): `bps` is the .bps image
 * (2-bit, base i of contig r at byte boff[r] + i/4, bits 2*(i%4)), clen/boff
 * the contig table (GDB_CONTIG, lib/GDB.h:29-35).  boff < 0 marks a contig
 * without sequence (skipped, as src/extract.c:101). */
int pga_gdb_load(pga_ctx *ctx, const uint8_t *bps, int64_t bps_bytes, int ncontig,
                 const int64_t *clen, const int64_t *boff);

/* Create_GDB (lib/GDB.c:442) on a FASTA text in host memory, parsed on the
 * device: the reader of lib/GDB.c:771-1057 with gap threshold `nthr` (the
 * reference's own callers pass 0: every N run followed by a base splits a
 * contig; a run shorter than nthr is otherwise filled with A's).  The result
 * is the context's GDB, as pga_gdb_load would leave it, with its base
 * frequencies set as Create_GDB sets GDB.freq (lib/GDB.c:1083-1086).
 * sizes6 (may be NULL) = {nscaff, ncontig, .bps bytes, header bytes,
 * maxctg, seqtot}.  The reference's errors are PGA_ERR_ARG with its message:
 * an empty text, a first line without '>', a last line without '\n', a
 * scaffold without sequence; NUL or non-ASCII bytes are refused too.  At
 * most 32767 contigs (PGA_ERR_LIMIT).  Soft masks (lower case, an ANO
 * argument of Create_GDB) are not produced. */
int pga_gdb_ingest_fasta(pga_ctx *ctx, const char *text, int64_t nbytes, int nthr, int64_t *sizes6);

/* The GDB made by pga_gdb_ingest_fasta, each array optional (NULL):
 * bps (sizes6[2] bytes), contigs4 (ncontig x {clen, boff, sbeg, scaf},
 * GDB_CONTIG lib/GDB.h:28-34), scaffolds4 (nscaff x {fctg, ectg, slen, hoff},
 * GDB_SCAFFOLD lib/GDB.h:36-41), headers (sizes6[3] bytes: each scaffold's
 * name ended by '\0', at hoff), counts4 (bases A C G T; filled gap bases
 * count as A). */
int pga_gdb_copy(pga_ctx *ctx, uint8_t *bps, int64_t *contigs4, int64_t *scaffolds4, char *headers,
                 int64_t *counts4);

/* Device times of the last pga_gdb_ingest_fasta, ms2 = {text upload, parse
 * (every kernel from the first header scan to the packed image)}. */
int pga_gdb_ingest_times(const pga_ctx *ctx, float *ms2);

/* Write_GDB (lib/GDB.c:1519) of the GDB made by pga_gdb_ingest_fasta:
 * tpath (<dir>/<root>.1gdb) and its hidden <dir>/.<root>.bps.  The .1gdb is
 * written in ONE's ASCII encoding; the reference's Read_GDB (lib/GDB.c:1171)
 * reads it.  srcpath is the FASTA's path as recorded in the file. */
int pga_gdb_write(pga_ctx *ctx, const char *tpath, const char *program, const char *version, const char *command,
                  const char *srcpath);

/* The writer behind pga_gdb_write, on host tables laid out as pga_gdb_copy's;
 * freq4 as GDB.freq.  Needs no device. */
int pga_write_1gdb(const char *tpath, const char *program, const char *version, const char *command,
                   const char *srcpath, const float *freq4, int nscaff, const int64_t *scaffolds4,
                   const char *headers, int64_t hdrtot, int ncontig, const int64_t *contigs4,
                   const uint8_t *bps, int64_t bps_bytes);

/* Record sizing of the loaded GDB (compute_record_sizing, src/record.c:18). */
int pga_record_sizing(const pga_ctx *ctx, int *position_bytes, int *contig_strand_bytes,
                      int *record_size);

/* ---- drop-in stages ------------------------------------------------------- */

/* extract_to_records (src/extract.h:40, src/extract.c:358): the records of
 * worker `worker_id` of `num_workers` (contig split of src/work_split.c:3),
 * in the reference's emission order, LCP byte 0.  *records is malloc'd with
 * one spare byte (msd_sort's sentinel, src/extract.c:268). */
int pga_extract_to_records(pga_ctx *ctx, int num_workers, int worker_id, uint8_t **records,
                           int64_t *count);

/* sort_records + recalc_all_lcps (src/sort.h:10-13), i.e. run_stage2 at world
 * size 1 (src/dsort.h:82): sorts `count` records of `record_size` bytes in
 * place by k-mer -- equal k-mers by payload -- and sets byte 0 to the bases
 * in common with the predecessor. */
int pga_sort_records(pga_ctx *ctx, uint8_t *records, int64_t count, int position_bytes,
                     int contig_strand_bytes);

/* build_kmer_adapter (src/kmer_adapter.h:46): entries (count x
 * (9 + position_bytes + contig_strand_bytes) bytes), the 2^24 cumulative
 * prefix counts and the largest prefix group, from sorted records. */
int pga_build_kmer_adapter(pga_ctx *ctx, const uint8_t *records, int64_t count, int position_bytes,
                           int contig_strand_bytes, uint8_t *entries, int64_t *cum,
                           int64_t *largest_group);

/* self_adaptamer_merge (src/fastga_pipeline.h:18) with one routing unit:
 * the N (same strand) and C seed byte streams (1 + 2*(posb+ctgb) bytes per
 * seed, malloc'd) and seeds per A contig (nbuck, cbuck: ncontig each). */
int pga_self_adaptamer_merge(pga_ctx *ctx, const uint8_t *entries, const int64_t *cum, int64_t count,
                             int position_bytes, int contig_strand_bytes, int freq, int ncontig,
                             uint8_t **nseeds, int64_t *nlen, uint8_t **cseeds, int64_t *clen,
                             int64_t *nbuck, int64_t *cbuck);

/* recalc_all_lcps (src/sort.c:38-57): byte 0 of each of `count` sorted
 * records (reference layout) becomes the number of leading bases its k-mer
 * shares with the previous record's (0 for the first), in place. */
int pga_recalc_lcps(pga_ctx *ctx, uint8_t *records, int64_t count, int position_bytes, int contig_strand_bytes);

/* reimport_thread + rmsd_sort (src/fastga_pipeline.c:1391-1450,
 * lib/RSDsort.c:292): `len` bytes of seeds -> swide-byte records, panel by A
 * contig, each panel sorted; panel_off (ncontig+1) gets record offsets.
 * comp = 0 for N seeds, 1 for C.  out needs (len/seed_bytes) * swide bytes,
 * swide = 2*dbyte + contig_strand_bytes + 2.  `len` must be a whole number
 * of seeds (PGA_ERR_ARG otherwise). */
int pga_reimport_sort(pga_ctx *ctx, const uint8_t *seeds, int64_t len, int position_bytes,
                      int contig_strand_bytes, int comp, int ncontig, int64_t amxpos, int dbyte,
                      uint8_t *out, int64_t *panel_off);

/* ---- resident pipeline ---------------------------------------------------- */

/* Extract + sort + LCP + k-mer table of the loaded GDB; want_entries = 0
 * skips writing the reference-format entries (the merge reads the device
 * records directly).  *count receives the record count. */
int pga_index_build(pga_ctx *ctx, int want_entries, int64_t *count);
int pga_index_copy_records(pga_ctx *ctx, uint8_t *records);           /* count x record_size */
/* GIXmake's output (notes/GIXmake_annotated.c:1529-1615) from the index built
 * with entries: <stem>.gix (header, the 2^24 cumulative prefix counts, the
 * contigs longest first -- what src/fastga_order_core.c:11 reads) and the
 * k-mer table in `nparts` parts <dir>/.<root>.ktab.1..nparts.  The part
 * boundaries (whole 10-bit panels, balanced by entries) and the order of equal
 * k-mers (by payload) are this library's; GIXmake picks both by sampling and
 * threads.  PGA_ERR_LIMIT when GIXmake's entry widths would differ from the
 * index's (a longest contig of exactly 256^k bases). */
int pga_index_write_gix(pga_ctx *ctx, const char *stem, int nparts);
/* The writer behind pga_index_write_gix, from host arrays: order[ncontig],
 * cum[2^24] (cumulative entries per prefix), nentries entries of
 * 9 + post_bytes + cont_bytes bytes.  Needs no device. */
int pga_write_gix(const char *stem, int nparts, int post_bytes, int cont_bytes, int ncontig, const int32_t *order,
                  const int64_t *cum, int64_t largest, int64_t nentries, const uint8_t *entries);
int pga_index_copy_entries(pga_ctx *ctx, uint8_t *entries, int64_t *cum, int64_t *largest_group);
/* The reader: a GIX on disk (written by GIXmake or pga_write_gix) as the
 * k-mer table view pga_self_adaptamer_merge takes (the reference reads the
 * header and contig order of the same file in fo_read_gix_perm,
 * src/fastga_order_core.c:11-52, and FastGA the parts).  hdr6 = {K, parts,
 * post_bytes, cont_bytes, frequency cutoff, ncontig}; *largest the largest
 * prefix group; *nentries.  With entries NULL only these are filled (the
 * sizes); otherwise also order[ncontig] (contigs longest first), cum[2^24]
 * and the entries (9 + post_bytes + cont_bytes bytes each), the parts back
 * to back, contigs numbered as in the GDB again (GIXmake numbers them by
 * their place in the order) and each part's first LCP byte taken to the
 * entry before it (GIXmake's part-by-part sort leaves another value there).
 * Runs of equal k-mers keep the file's order.  Needs no device. */
int pga_read_gix(const char *stem, int *hdr6, int32_t *order, int64_t order_cap, int64_t *cum, int64_t *largest,
                 int64_t *nentries, uint8_t *entries, int64_t entries_cap);

/* Adaptamer merge of the built index: seeds stay in HBM. */
int pga_merge(pga_ctx *ctx, int freq, int64_t *nseeds, int64_t *cseeds);
int pga_seeds_copy(pga_ctx *ctx, int comp, uint8_t *seeds, int64_t *buck);

/* Seeds of unit comp (0 = N, 1 = C) from the host into the context, as
 * pga_merge would leave them: `len` bytes of seeds in the reference layout
 * (1 + 2*(posb+ctgb) bytes each, the loaded GDB's field widths), the
 * received seed buffers pair_sort_search starts from (Recv_N_Data /
 * Recv_C_Data, src/fastga_pipeline.c:1793-1806).  The first load after a
 * merge (or none) empties the other unit until it is loaded too. */
int pga_seeds_load(pga_ctx *ctx, int comp, const uint8_t *seeds, int64_t len);

/* Reimport + diagonal sort of unit comp (0 = N, 1 = C) in HBM. */
int pga_diag_sort(pga_ctx *ctx, int comp, int *swide, int64_t *count);
int pga_diag_copy(pga_ctx *ctx, int comp, uint8_t *records, int64_t *panel_off);

/* ---- alignment ------------------------------------------------------------ */

/* Base frequencies of the GDB (GDB.freq, lib/GDB.h:67); they set the
 * aligner's scoring tables (New_Align_Spec, lib/align.c:222).  Without this
 * call they are computed from the loaded sequence as the GDB stores them. */
int pga_gdb_set_freq(pga_ctx *ctx, const float *freq4);

/* pair_sort_search's alignment half (src/fastga_pipeline.c:1686-1892 with
 * fastga_order's self-pair entry values, src/fastga_order.c:276): chains and
 * Local_Alignment (lib/align.c:1423) over every (anchor, partner) pair of the
 * N and C units, the per-pair elimination / entwine step, and la_sort's
 * order (aread, abpos, bread, comp).  Runs pga_diag_sort on both units if
 * needed.  *nalign = surviving alignments. */
int pga_align(pga_ctx *ctx, int64_t *nalign);

/* FastGA's thread ranges over its contig order, the split pga_align's
 * self-pair rules use (fo_compute_ranges, src/fastga_order_core.c:50-140):
 * clen_pos and seeds_pos by order position (lengths, N-unit seed counts),
 * npost the GDB's total bases, swide the sorted-seed record width, nthreads
 * FastGA's thread count (32 in the reference's driver).  Fills
 * range_start[x] = the first position of x's range.  Host only. */
int pga_fastga_ranges(int n, const int64_t *clen_pos, int64_t npost, const int64_t *seeds_pos, int64_t swide,
                      int nthreads, int *range_start);

/* How pga_align spreads large pairs of two different contigs over warps: it
 * cuts such a pair into ranges of about range_seeds seeds at band
 * boundaries, aligns the ranges on different warps (a pair's band blocks are
 * independent) and finishes the pair from the ranges' candidates in order;
 * the result is the same for every setting.  0 (default): automatic; -1: never
 * split; n > 0: ranges of n seeds.  No counterpart in the reference (one
 * thread runs each pair there). */
int pga_align_set_ranges(pga_ctx *ctx, int64_t range_seeds);

/* Where the last pga_align's warps spent their time: prof2[0] = SM cycles
 * inside Local_Alignment calls, prof2[1] = SM cycles in the pairs' finishing
 * steps, each summed over warps (the rest of a task's cycles is the chain
 * scan and its bookkeeping). */
int pga_align_profile(const pga_ctx *ctx, int64_t *prof2);
/* Tuning, no counterpart in the reference: which build of the alignment
 * kernel runs -- 2 (255 registers, two CTAs per SM: best when the launch is
 * bounded by its longest alignments), 3 (168 registers, three CTAs per SM),
 * 4 (128 registers, four) or 5 (96 registers, five CTAs per SM: best for
 * launches of many pairs); 0 (the default) picks 5 above 2^20 pairs, else 2.
 * The alignments are the same either way. */
int pga_align_set_build(pga_ctx *ctx, int ctas_per_sm);

/* Tuning, no counterpart in the reference: when one Local_Alignment call of
 * the alignment launch passes this many wave steps (in one direction), the
 * other warps on its SM take no new pair task, so that the long call --
 * which bounds the launch -- soon has the SM to itself; the remaining tasks
 * go to the other SMs.  0 turns this off;
 * -1 (the default) is 20000 for launches of the two-CTA build and off for
 * the builds of three to five CTAs per SM (launches of more than 2^20
 * pairs, bounded by throughput).  The alignments are the same for every
 * value. */
int pga_align_set_long_waves(pga_ctx *ctx, int waves);

/* Tuning, no counterpart in the reference: the width in bits (18..22) of the
 * first-level digit of pga_index_build's two-level sort; 0 (the default)
 * takes 18 unless digits would then average more than 8192 records.  The
 * index is the same for every width. */
int pga_index_set_digit_bits(pga_ctx *ctx, int bits);

/* ---- Served form: a resident target and query requests ------------------
 * No counterpart in the reference, which runs one GDB per job.  A request's
 * results are, bit for bit, those of the plain path on the GDB that
 * pga_gdb_ingest_fasta makes of the target's FASTA text followed by the
 * query's (every pair of that GDB is aligned: the frequency cutoff and
 * FastGA's self-pair order both depend on all of its contigs). */

/* Moves ctx's GDB (ingested with pga_gdb_ingest_fasta) and its index
 * (pga_index_build) into a new resident target; ctx is left with no GDB.  The
 * target is read-only: any number of contexts of the same device may serve
 * requests against it at once, each on its own stream. */
int pga_target_create(pga_ctx *ctx, pga_target **out);
/* The same, with a record of the target's own Local_Alignment calls: ctx
 * first runs the target's GDB through the adaptamer merge (FREQ = freq) and
 * the alignment, logging every call -- its inputs (the two contigs, the
 * orientation, low, hgh, anti, lbord, hbord) and its result (the path and
 * its trace points) -- and the target keeps them in a table.  pga_align on a
 * request's GDB (pga_serve_load) then answers a call on two target contigs
 * whose inputs are in the table with the recorded result instead of running
 * the wave loop: the same result, since a call's result is a function of its
 * inputs, the two contigs' bases and the scoring tables, and the table is
 * used only when the request's scoring tables are the target run's. */
int pga_target_create_reuse(pga_ctx *ctx, int freq, pga_target **out);
void pga_target_destroy(pga_target *t);
/* info4 = {contigs, bases, index records, device bytes held}. */
int pga_target_info(const pga_target *t, int64_t *info4);
/* The last pga_align's use of a target's record of calls: stats4 = {used
 * (0/1), calls answered from the record, calls made in all, why it was not
 * used: 0 it was, or no target / 1 the target has no record / 3 the scoring
 * tables differ (base composition)}. */
int pga_align_reuse_stats(const pga_ctx *ctx, int64_t *stats4);

/* A request: ctx's GDB becomes GDB(target's text, query text) -- the query
 * parsed on the device with the target's gap threshold, its contigs and
 * scaffolds numbered after the target's -- and its index is built from the
 * query's records alone, sorted, and merged into the target's resident
 * sorted records (k_union_rank) instead of sorting both.  Then pga_merge,
 * pga_align and the writers run as for any GDB.  sizes6 as
 * pga_gdb_ingest_fasta gives it for the combined GDB; count = index records.
 * The query's errors are pga_gdb_ingest_fasta's; PGA_ERR_LIMIT when the two
 * together pass 32767 contigs or scaffolds. */
int pga_serve_load(pga_ctx *ctx, const pga_target *t, const char *query, int64_t nbytes, int want_entries,
                   int64_t *sizes6, int64_t *count);

/* The alignments in la_sort order: per alignment 9 ints (aread abpos aepos
 * bread bbpos bepos comp diffs tlen), trace_off (nalign+1) and the trace
 * bytes (uint8 pairs: differences, b-delta per 100-base A interval, as
 * Compress_TraceTo8 leaves them, lib/align.c:3892). */
int pga_align_copy(pga_ctx *ctx, int32_t *recs9, int64_t *trace_off, uint8_t *trace);

/* [0] pairs [1] self pairs [2] Local_Alignment calls [3] SM cycles of the
 * longest warp task (a pair, or a band range of a large pair) [4] alignments
 * [5] self-pair rounds [6] SM cycles of all tasks [7] Local_Alignment calls
 * of the longest task */
int pga_align_stats(const pga_ctx *ctx, int64_t *stats8);

/* Host wall-clock split of the last pga_align, in ms: [0] set-up (diagonal
 * sort if needed, sequences, pair lists) [1] pairs of two contigs and all C
 * pairs (one launch plus the band-range finish) [2] self pairs (rounds of
 * FastGA's order) [3] la_sort order and read-back.  No counterpart in the
 * reference. */
int pga_align_times(const pga_ctx *ctx, float *ms4);

/* Work of the last pga_align: [0] wave steps of all Local_Alignment calls
 * (after each call's first wave), [1] their diagonal updates ("cells", the
 * unit of forward_wave / reverse_wave, lib/align.c:639-753), [2]
 * Local_Alignment calls, [3] warp tasks.  No counterpart in the reference. */
int pga_align_work(const pga_ctx *ctx, int64_t *work4);

/* ---- Local_Alignment on request lists -------------------------------------------- */

/* Local_Alignment (lib/align.c:1423-1576) for n independent requests on the
 * loaded contigs, as align_contigs calls it (src/fastga_pipeline.c:720-775):
 * request i is 8 ints "a b comp low hgh anti lbord hbord" -- contig a
 * (reverse-complemented when comp) against contig b, diagonal band [low, hgh]
 * at antidiagonal anti, borders lbord / hbord (-1 = none); the band's start
 * points ((anti+k)/2, (anti-k)/2) must lie in the contigs (PGA_ERR_ARG
 * otherwise: the reference reads outside its buffers there).  Trace spacing 100;
 * the scoring tables follow the GDB's base frequencies (pga_gdb_set_freq) as
 * New_Align_Spec(0.7, 100, freq, 0).  One warp per request.  *ntrace = total
 * trace values of the results. */
int pga_local_alignment(pga_ctx *ctx, int64_t n, const int32_t *req8, int64_t *ntrace);

/* The results of the last pga_local_alignment, in request order: path7 (7
 * ints each: abpos aepos bbpos bepos diffs tlen status, status 0 or a work
 * space overflow code), trace_off (n+1), trace (the tlen uint16 values of
 * each path: diffs, b-delta per trace interval, as Local_Alignment leaves
 * them before Compress_TraceTo8). */
int pga_local_alignment_copy(pga_ctx *ctx, int32_t *path7, int64_t *trace_off, uint16_t *trace);

/* ---- the .1aln file ------------------------------------------------------------ */

/* la_merge's output file (src/fastga_pipeline.c:1616-1656: open_Aln_Write,
 * Write_Skeleton, Write_Aln_Overlap, Write_Aln_Trace; lib/alncode.c:239-305,
 * lib/GDB.c:2059-2086), as an ASCII ONE file of type "aln" that ONE readers
 * (open_Aln_Read, ALNtoPAF) read like the reference's binary one: header with
 * provenance (program, version, command, date), references db_name (1) and
 * cwd (3, may be NULL), the trace spacing, the GDB skeleton (per scaffold
 * its name, then G gap / C contig lengths; contigs of scaffold s are
 * [scaff_fctg[s], scaff_fctg[s+1]), at contig_sbeg within the scaffold), then
 * the alignments as pga_align_copy gives them: recs9 (aread abpos aepos
 * bread bbpos bepos comp diffs tlen), trace_off, trace.  Host only. */
int pga_write_1aln(const char *path, const char *program, const char *version, const char *command,
                   const char *db_name, const char *cwd, int tspace, int nscaff, const char *const *scaff_name,
                   const int64_t *scaff_len, const int32_t *scaff_fctg, const int64_t *contig_sbeg,
                   const int64_t *contig_len, int64_t nalign, const int32_t *recs9, const int64_t *trace_off,
                   const uint8_t *trace);

/* The same file in ONE's binary encoding, the one the reference's
 * open_Aln_Write asks ONElib for (lib/alncode.c:251, isBinary true): the
 * same header up to the line definitions, then "$ 0" (little-endian), the
 * lines as one code byte and their fields (variable-length integers,
 * difference-coded integer lists), and a footer with the counts, list
 * maxima and totals, per-object statistics and the objects' byte index that
 * ONE readers use.  Trace lists are coded with a length-limited Huffman
 * code built from all of them (stored in the footer as ONElib stores its
 * codecs) wherever that is shorter; ONElib builds its code from a type's
 * first 100,000 list bytes.  Host only. */
int pga_write_1aln_binary(const char *path, const char *program, const char *version, const char *command,
                          const char *db_name, const char *cwd, int tspace, int nscaff,
                          const char *const *scaff_name, const int64_t *scaff_len, const int32_t *scaff_fctg,
                          const int64_t *contig_sbeg, const int64_t *contig_len, int64_t nalign,
                          const int32_t *recs9, const int64_t *trace_off, const uint8_t *trace);

/* The same for the alignments of the last pga_align, with the loaded
 * contigs' lengths: ASCII, or binary (pga_align_write_1aln_binary). */
int pga_align_write_1aln(pga_ctx *ctx, const char *path, const char *program, const char *version,
                         const char *command, const char *db_name, const char *cwd, int nscaff,
                         const char *const *scaff_name, const int64_t *scaff_len, const int32_t *scaff_fctg,
                         const int64_t *contig_sbeg);
int pga_align_write_1aln_binary(pga_ctx *ctx, const char *path, const char *program, const char *version,
                                const char *command, const char *db_name, const char *cwd, int nscaff,
                                const char *const *scaff_name, const int64_t *scaff_len,
                                const int32_t *scaff_fctg, const int64_t *contig_sbeg);

/* ---- seed diagonal sort without device allocation ---------------------------- */

/* No counterpart in the reference: the reference runs on the host and never
 * meets this constraint.  The same result as pga_reimport_sort, for callers
 * that may not call cudaMalloc -- for instance a program living inside
 * another framework's device memory pool (PyTorch's caching allocator, a
 * serving runtime's arena) that owns the GPU memory it may use.  The caller
 * passes device buffers it already owns: `seeds_dev` (len bytes of seeds),
 * `out_dev` ((len/seed_bytes) * swide bytes) and `panel_off_dev`
 * (ncontig+1 int64); no context is needed.  All other work space is one
 * fixed array compiled into the library (about 12 MB, held on every GPU that
 * loads it until the process exits).  At most 262,144 seeds per call
 * (PGA_ERR_LIMIT beyond); `len` must be a whole number of seeds
 * (PGA_ERR_ARG otherwise).  The first call on a device looks the array's
 * address up for that device (and looks it up again after the device's
 * context was re-created, e.g. by cudaDeviceReset).  The call cannot be
 * captured into a CUDA graph: it synchronizes `stream` (a cudaStream_t, NULL
 * for the default stream) once, midway; the last kernels are left queued on
 * it.
 * Calls share the array: calls that overlap on the GPU (several host
 * threads or streams) race.  Returns PGA_OK, PGA_ERR_ARG, PGA_ERR_LIMIT or
 * PGA_ERR_CUDA. */
int pga_reimport_sort_noalloc(const uint8_t *seeds_dev, int64_t len, int position_bytes,
                              int contig_strand_bytes, int comp, int ncontig, int64_t amxpos, int dbyte,
                              uint8_t *out_dev, int64_t *panel_off_dev, void *stream);

#ifdef __cplusplus
}
#endif

#endif
