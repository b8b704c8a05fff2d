/* The reference's own stage entry points, with its exact signatures, running
 * on a B200 through libpga_b200.so.
 *
 * A build of the reference's driver (src/pga-mpi-merge.c) links
 * distributedpanga_b200/dropin/pga_dropin.c and libpga_b200.so in place of
 * src/extract.c, src/sort.c, src/kmer_adapter.c and src/fastga_pipeline.c;
 * every other file of the driver's build (src/dsort.c, src/record.c,
 * src/seed_buffer.c, src/fastga_order.c, lib/ ...) and the driver's flow are
 * unchanged.  This header is compiled with the reference's own include paths
 * (its lib/ and src/ directories and an mpi.h): the types below are the
 * reference's, declared there.
 *
 * Scope: one process (world size 1, NTHREADS 1), one GPU (device 0, or the
 * PGA_DEVICE environment variable).  The driver's alignment parameters must
 * be its defaults (KMER 40, CHAIN_BREAK 2000, CHAIN_MIN 170, ALIGN_MIN 100,
 * ALIGN_RATE 0.3), which the device code is built with; FREQ is read at run
 * time.  Errors end the process with a message and exit(1), as the
 * reference's stages do.
 */
#ifndef PGA_DROPIN_H
#define PGA_DROPIN_H

#include <mpi.h>
#include "GDB.h"
#include "extract.h"
#include "record.h"
#include "sort.h"
#include "kmer_adapter.h"
#include "fastga_pipeline.h"

/* src/extract.h:40 (src/extract.c:358): the closed-syncmer records of worker
 * worker_id's contigs (compute_work_split's range), appended to buf (which
 * record_buffer_init made, with its +1 sentinel byte); g_extract_stats gets
 * the contigs and bases scanned. */
void extract_to_records(GDB *gdb, int num_workers, int worker_id, RecordBuffer *buf);
void extract_stats_reset(void);          /* src/extract.h:58 */
/* src/extract.h:37-38: the record buffer (capacity in records, +1 sentinel
 * byte) */
void record_buffer_init(RecordBuffer *b, RecordSizing sizing);
void record_buffer_free(RecordBuffer *b);
/* src/extract.h:24-26: the same records as tuples (contig, position, strand,
 * k-mer bytes), appended to buf */
void tuple_buffer_init(TupleBuffer *b);
void tuple_buffer_free(TupleBuffer *b);
void extract_to_tuples(GDB *gdb, int num_workers, int worker_id, TupleBuffer *buf);

/* src/sort.h:10-16 (src/sort.c:16-115): sort_records orders the records by
 * k-mer (equal k-mers by payload) and leaves byte 0 the bases-in-common LCP;
 * recalc_all_lcps rewrites byte 0 the same way; simple_kmer_lcp_bases counts
 * the leading bases two k-mers share. */
void sort_records(RecordBuffer *buf);
void recalc_all_lcps(RecordBuffer *buf);
int simple_kmer_lcp_bases(const uint8_t *a, const uint8_t *b, int kbytes);

/* src/kmer_adapter.h:46-57 (src/kmer_adapter.c:6-162): the sorted records
 * as the merge's k-mer table (entries, the 2^24 cumulative prefix counts,
 * the largest prefix group), and its cursor operations. */
int build_kmer_adapter(const RecordBuffer *buffer, KmerStreamAdapter *kmer_table, PayloadLayout *payload_layout);
void free_kmer_adapter(KmerStreamAdapter *kmer_table, PayloadLayout *payload_layout);
void adapter_First_Kmer_Entry(KmerStreamAdapter *kmer_table);
void adapter_Next_Kmer_Entry(KmerStreamAdapter *kmer_table);
void adapter_GoTo_Kmer_Index(KmerStreamAdapter *kmer_table, int64 i);
KmerStreamAdapter *adapter_Clone_Kmer_Stream(KmerStreamAdapter *kmer_table);
void adapter_Free_Kmer_Stream(KmerStreamAdapter *kmer_table);
uint8 *adapter_Current_Entry(KmerStreamAdapter *kmer_table, uint8 *ent);

/* src/fastga_pipeline.h:18 (src/fastga_pipeline.c:418-499): the adaptamer
 * merge of the table under FREQ; seeds go to N_SeedUnits / C_SeedUnits
 * (unit = RankForPair of the pair) and per-A-contig counts to
 * N_Units[0].buck / C_Units[0].buck. */
void self_adaptamer_merge(KmerStreamAdapter *kmer_table, PayloadLayout *payload_layout, int64 g1len);

/* src/fastga_pipeline.h:19 (src/fastga_pipeline.c:1686-1842): reimport,
 * diagonal sort, chaining and Local_Alignment of the received seeds
 * (Recv_N_Data / Recv_C_Data, freed here), in FastGA's pair order, written
 * as $SORT_PATH/$ALGN_UNIQ.1aln with gdb1's skeleton; Pair_Search_Stats
 * gets the stage times.  Self_Order (installed by fastga_order_setup) is not
 * consulted: the library computes FastGA's self-pair entry values itself. */
void pair_sort_search(GDB *gdb1, GDB *gdb2);

#endif
