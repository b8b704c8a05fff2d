/* CPU restatement of DistributedPanGA's FastGA alignment path, stages
 * extract -> index sort + LCP -> k-mer table view -> adaptamer seed merge ->
 * seed reimport + diagonal sort, and of the GDB's FASTA reader.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  It is pinned by tests against the reference's own known
 * answers (tests/unit/test_extract.c, tests/unit/test_lcp_sort.c,
 * tests/unit/test_adapter.c) and against dumps of the reference pipeline
 * compiled from source (oracle/_ref).
 *
 * Byte layouts are the reference's:
 *   record  (src/record.h:8-26)        [LCP][k-mer 10, MSB-first][mask 0][pos P LE][ctg|strand C LE]
 *   entry   (src/kmer_adapter.c:15-18) [k-mer bytes 3..9][mask 0][LCP][payload P+C]
 *   seed    (src/fastga_pipeline.c:391-397) [plen][A payload, strand cleared][B payload]
 *   sorted seed record (src/fastga_pipeline.c:1434-1446)
 *           [lcp][diag & 63][anti DBYTE LE][diag >> 6 DBYTE LE][jcont C LE]
 */
#ifndef PGA_ORACLE_H
#define PGA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The syncmer hash's 256-entry 4-mer table (src/tables.c:5-22). */
const uint8_t *orc_tmap(void);

/* Record sizing from the contig table (src/record.c:18-37). */
void orc_record_sizing(int ncontig, int64_t maxctg, int *posb, int *ctgb, int *rsize);

/* Closed-(12,8)-syncmer extraction of every contig (src/extract.c:85-249,
 * src/pack.c:29-78), records appended in the reference's emission order
 * (contig, then j, forward before reverse complement).  `bps` is the GDB's
 * 2-bit sequence file: base i of contig r at byte boff[r] + i/4, bits
 * 2*(i%4) (lib/gene_core.c:359-378).  Returns the record count; writes at
 * most `cap` records when `out` is not NULL. */
int64_t orc_extract(const uint8_t *bps, int ncontig, const int64_t *clen, const int64_t *boff,
                    int posb, int ctgb, uint8_t *out, int64_t cap);

/* Sort records by k-mer, equal k-mers by their payload bytes read as one
 * little-endian integer (contig|strand most significant, then position),
 * then overwrite byte 0 with the bases-in-common LCP to the predecessor
 * (src/sort.c:16-115).  The reference leaves equal k-mers in an unspecified
 * order; this order is the canonical one the CUDA path also produces. */
void orc_sort_records(uint8_t *rec, int64_t n, int rsize);

/* Bases in common of two packed 40-mers, [0,40] (src/sort.c:16-32). */
int orc_lcp_bases(const uint8_t *a, const uint8_t *b);

/* The k-mer table view (src/kmer_adapter.c:6-96): entries and the 2^24
 * cumulative prefix counts (cum[p] = #entries with 24-bit prefix <= p).
 * Returns the largest prefix group's size. */
int64_t orc_build_adapter(const uint8_t *rec, int64_t n, int rsize, int posb, int ctgb,
                          uint8_t *entries, int64_t *cum);

/* FastGA's self adaptamer merge, restated as the reference's sequential walk
 * over each 24-bit prefix group (src/fastga_pipeline.c:245-412) with one
 * routing unit (world size 1).  Seeds go to the N buffer when both k-mers
 * are on the same strand, else to C.  Returns 0, or -1 when a buffer is
 * too small (its required length is still reported).  nbuck/cbuck
 * (ncontig each) count seeds per A contig. */
int orc_merge(const uint8_t *entries, const int64_t *cum, int64_t n, int ebytes, int posb, int ctgb,
              int freq, int ncontig,
              uint8_t *nseed, int64_t ncap, int64_t *nlen,
              uint8_t *cseed, int64_t ccap, int64_t *clen_out,
              int64_t *nbuck, int64_t *cbuck);

/* Seed reimport and diagonal sort (src/fastga_pipeline.c:1391-1450,
 * lib/RSDsort.c:292-377): every seed becomes one swide-byte record in the
 * panel of its A contig, and each panel is sorted on all swide bytes read
 * from the last byte backwards.  comp = 0 for N seeds, 1 for C seeds.
 * `panel_off` (ncontig+1) receives the record offset of every panel.
 * Returns swide. */
int orc_reimport_sort(const uint8_t *seeds, int64_t len, int posb, int ctgb, int comp,
                      int ncontig, int64_t amxpos, int dbyte,
                      uint8_t *out, int64_t *panel_off);

/* swide and DBYTE for a contig set (src/pga-mpi-merge.c:415-425,
 * src/fastga_pipeline.c:1736). */
void orc_diag_sizing(int64_t maxctg, int ctgb, int *dbyte, int *swide);

/* Create_GDB's FASTA reader (lib/GDB.c:771-1057, base table lib/GDB.c:350-367)
 * on an in-memory text, with nthr as given (the reference's own callers pass
 * 0, lib/GDB.c:1662):
 *   scf4  nscaff x {fctg, ectg, slen, hoff}   (GDB_SCAFFOLD, lib/GDB.h:36-43)
 *   ctg4  ncontig x {clen, boff, sbeg, scaf}  (GDB_CONTIG, lib/GDB.h:28-34)
 *   hdr   the header bytes, each ended by '\0'
 *   bps   the 2-bit image, LSB-first, each contig from a fresh byte
 *   sizes {nscaff, ncontig, bps bytes, hdrtot, maxctg, seqtot}
 *   count bases per value A C G T (filled gap bases count as A)
 * Returns 0; -1 for an input the reference rejects or cannot read (message in
 * err); -2 when a capacity is too small. */
int orc_fasta_gdb(const char *text, int64_t n, int nthr,
                  int64_t *scf4, int64_t scf_cap, int64_t *ctg4, int64_t ctg_cap,
                  char *hdr, int64_t hdr_cap, uint8_t *bps, int64_t bps_cap,
                  int64_t *sizes6, int64_t *count4, char *err, int errlen);

#ifdef __cplusplus
}
#endif

#endif
