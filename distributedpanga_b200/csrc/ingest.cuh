// GDB ingest: FASTA text -> 2-bit sequence image + scaffold/contig tables,
// the result of Create_GDB's FASTA reader (lib/GDB.c:771-1057).
//
// Device layout while a text is parsed:
//   text   n bytes (+64 zero bytes)          the FASTA as given
//   mask   1 bit per text byte               set on header lines, '\n' included
//   seq    G bytes (+64)                     every sequence character in text
//                                            order, value 0..3 (base) or 4 (N),
//                                            bit 3 set on a scaffold's first
//   runs   rs/re per maximal N run of seq    [start, end) in seq positions
// and the tables (seq positions are global; sbeg/slen are derived):
//   hstart/hend  per scaffold: '>' and its line's '\n' in text
//   sstart       per scaffold (+1): first seq position; sstart[nscaff] = G
//   cstart/cend  per contig: its seq interval
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pga {

constexpr int FA_THREADS = 256;
constexpr int FA_BYTES = 16;                       // text bytes per thread
constexpr int FA_TILE = FA_THREADS * FA_BYTES;     // 4096 text bytes per block

// Status words (u64) written by the parse kernels.
enum FaStatusWord {
  FA_BAD = 0,        // min text position of a NUL or non-ASCII byte (~0 = none)
  FA_EMPTY = 1,      // min scaffold without any sequence character (~0 = none)
  FA_ALLN = 2,       // min scaffold whose sequence is all N (~0 = none)
  FA_COUNT = 3,      // 4 words: bases per value 0..3 (filled gap bases not included)
  FA_FILL = 7,       // bases of gaps filled with A (shorter than nthr)
  FA_MAXCTG = 8,     // longest contig
  FA_NSTATUS = 16
};

cudaError_t fa_init_status(unsigned long long *status, cudaStream_t st);

// Header starts: '>' at a line start.  Also finds NUL / non-ASCII bytes.
cudaError_t fa_count_headers(const uint8_t *text, int64_t n, int64_t *cnt, unsigned long long *status,
                             cudaStream_t st);
cudaError_t fa_write_headers(const uint8_t *text, int64_t n, const int64_t *off, int64_t *hstart,
                             cudaStream_t st);
// Per header: its line end, the text after '>' and white space, and that
// text's length + 1 (the header block entry with its '\0').
cudaError_t fa_header_lines(const uint8_t *text, const int64_t *hstart, int nh, int64_t *hend, int64_t *htext,
                            int64_t *hlen1, cudaStream_t st);
cudaError_t fa_copy_headers(const uint8_t *text, const int64_t *htext, const int64_t *hlen1, const int64_t *hoff,
                            int nh, char *hdr, cudaStream_t st);
cudaError_t fa_paint_headers(const int64_t *hstart, const int64_t *hend, int nh, uint32_t *mask, cudaStream_t st);

// Sequence characters: the bytes neither on a header line nor '\n'.
cudaError_t fa_count_seq(const uint8_t *text, int64_t n, const uint32_t *mask, int64_t *cnt, cudaStream_t st);
cudaError_t fa_write_seq(const uint8_t *text, int64_t n, const uint32_t *mask, const int64_t *off,
                         const int64_t *hend, int nh, uint8_t *seq, int64_t *sstart,
                         unsigned long long *status, cudaStream_t st);
cudaError_t fa_flag_scaffolds(uint8_t *seq, const int64_t *sstart, int nh, unsigned long long *status,
                              cudaStream_t st);

// Maximal N runs of each scaffold's sequence.
cudaError_t fa_count_runs(const uint8_t *seq, int64_t G, int64_t *cnt_start, int64_t *cnt_end, cudaStream_t st);
cudaError_t fa_write_runs(const uint8_t *seq, int64_t G, const int64_t *off_start, const int64_t *off_end,
                          int64_t *rs, int64_t *re, cudaStream_t st);
cudaError_t fa_classify_runs(const int64_t *rs, const int64_t *re, int64_t R, const int64_t *sstart, int nh,
                             int nthr, int64_t *is_split, int32_t *rscaf, int64_t *trail,
                             unsigned long long *status, cudaStream_t st);

// Contig intervals from the scaffolds and the splitting runs.
// scf4: per scaffold {fctg, ectg, slen, hoff} (GDB_SCAFFOLD, lib/GDB.h:36-41).
cudaError_t fa_scaffolds(const int64_t *sstart, int nh, const int64_t *rs, int64_t R, const int64_t *sr,
                         int64_t nsplit, const int64_t *trail, const int64_t *hoff, int64_t *scf4,
                         int64_t *cstart, int64_t *cend, int32_t *cscaf, cudaStream_t st);
cudaError_t fa_splits(const int64_t *rs, const int64_t *re, int64_t R, const int64_t *is_split, const int64_t *sr,
                      const int32_t *rscaf, int64_t *cstart, int64_t *cend, int32_t *cscaf, cudaStream_t st);
// clen, sbeg and the byte count of every contig; longest contig.
cudaError_t fa_contigs(int nc, const int64_t *cstart, const int64_t *cend, const int32_t *cscaf,
                       const int64_t *sstart, int64_t *clen, int64_t *sbeg, int64_t *nbytes,
                       unsigned long long *status, cudaStream_t st);
// The 2-bit image: base i of contig c at byte boff[c] + i/4, bits 2*(i%4);
// boff has nc + 1 entries (boff[nc] = image bytes).  Writes whole 4-byte
// words up to round_up(boff[nc], 4).
cudaError_t fa_pack(const uint8_t *seq, int nc, const int64_t *boff, const int64_t *cstart, const int64_t *clen,
                    uint8_t *bps, cudaStream_t st);

}  // namespace pga
