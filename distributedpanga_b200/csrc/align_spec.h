// Host-side construction of the aligner's scoring tables: New_Align_Spec
// (lib/align.c:222-268) with ave_corr = 1 - ALIGN_RATE = 0.7, trace spacing
// 100 and reach 0, as the reference's search_seeds calls it
// (src/fastga_pipeline.c:1101).
#pragma once
#include <stdint.h>

namespace pga {
namespace aln {

// The tip-trimming tables: for every TRIM_LEN-bit match/mismatch history x,
// score[x] is its score (match +mscore, mismatch -dscore, in 1/1000 units)
// and table[x] its score minus the best prefix score.
inline void fill_trim_tables(int bit, int prefix, int score, int max, int mscore, int dscore, int16_t *score_t,
                             int16_t *table_t) {
  if (bit >= 15) {
    table_t[prefix] = (int16_t)(score - max);
    score_t[prefix] = (int16_t)score;
  } else {
    if (score > max) max = score;
    fill_trim_tables(bit + 1, prefix << 1, score - dscore, max, mscore, dscore, score_t, table_t);
    fill_trim_tables(bit + 1, (prefix << 1) | 1, score + mscore, max, mscore, dscore, score_t, table_t);
  }
}

// freq: the GDB's base frequencies (float, as stored).  Fills score_t and
// table_t (32768 entries each) and returns ave_path.
inline int build_align_spec(const float *freq, int16_t *score_t, int16_t *table_t) {
  static const double bias_factor[10] = {.690, .690, .690, .690, .780, .850, .900, .933, .966, 1.000};
  const double ave_corr = 1. - 0.3;
  float fm = freq[0] + freq[3];
  double match = fm;
  if ((match <= 0.) == (match > 0.)) match = .5;
  if (match > .5) match = 1. - match;
  int bias = (int)((match + .025) * 20. - 1.);
  if (match < .2) bias = 3;
  int ave_path = (int)(60 * (1. - bias_factor[bias] * (1. - ave_corr)));
  int mscore = (int)(1000 * bias_factor[bias] * (1. - ave_corr));
  int dscore = 1000 - mscore;
  fill_trim_tables(0, 0, 0, 0, mscore, dscore, score_t, table_t);
  return ave_path;
}

}  // namespace aln
}  // namespace pga
