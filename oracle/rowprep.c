/* Host row preparation of sequence queries, restated for the oracle (TEST
 * INFRASTRUCTURE ONLY): the composition-bias correction and the low-complexity
 * mask that the reference applies to a sequence query's score rows before
 * scoring (src/search.rs:432-455).  The GPU kernels take whatever int32 rows
 * they are given; these functions exist so that the oracle can rebuild the
 * exact rows behind the reference's own recorded search outputs
 * (tests/data/v1_fixture_k2.v03.m8) and be checked against them.
 *
 * Floating point is binary64 with libm's log2, as the reference computes it
 * with Rust's f64 (which calls the same libm on Linux). */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "oracle.h"

#define OR_ALPHA 21
#define OR_PROFILE_AA 20

static int32_t round_half_away(double x) {
  /* src/compbias.rs:73-80 */
  return x >= 0.0 ? (int32_t)floor(x + 0.5) : -(int32_t)floor(-x + 0.5);
}

/* local_bias_correction_mode, src/compbias.rs:38-70: for query position i with
 * residue a, delta_i = sum_b p_back[b] s(a,b) - (1/|W_i|) sum_{j in W_i, j != i} s(a, q_j)
 * over the window [i-20, i+20) clipped to the query, rounded half away from zero.
 * score: the 21x21 integer matrix (row-major, codes 0..20); p_back: 20 entries. */
void or_comp_bias(const uint8_t* q, uint32_t n, const int32_t* score, const double* p_back, int penalize_only,
                  int32_t* out) {
  double expected[OR_ALPHA];
  for (int a = 0; a < OR_ALPHA; ++a) {
    double e = 0.0;
    for (int b = 0; b < OR_PROFILE_AA; ++b) e += p_back[b] * (double)score[a * OR_ALPHA + b];
    expected[a] = e;
  }
  const uint32_t half = 20; /* WINDOW / 2, src/compbias.rs:28 */
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t lo = i > half ? i - half : 0;
    const uint32_t hi = i + half < n ? i + half : n;
    const int a = q[i] < OR_ALPHA ? q[i] : OR_ALPHA - 1;
    int64_t sum = 0;
    for (uint32_t j = lo; j < hi; ++j)
      if (j != i) sum += score[a * OR_ALPHA + (q[j] < OR_ALPHA ? q[j] : OR_ALPHA - 1)];
    const double wl = (double)(hi - lo);
    const double delta = expected[a] - (double)sum / wl;
    const int32_t d = round_half_away(delta);
    out[i] = penalize_only && d > 0 ? 0 : d;
  }
}

/* low_complexity_mask_into, src/mask.rs:68-128: Shannon entropy of the residue
 * composition of every w-residue window (a sliding sum of c*log2(c)); a window
 * at or below locut triggers, the segment extends over neighbouring windows at
 * or below hicut, and every position of the covered windows is masked.
 * Returns the number of masked positions. */
uint32_t or_low_complexity_mask(const uint8_t* seq, uint32_t n, uint32_t w, double locut, double hicut,
                                uint8_t* mask) {
  for (uint32_t i = 0; i < n; ++i) mask[i] = 0;
  if (w < 2 || n < w) return 0;
  double* clog = (double*)calloc(w + 1, sizeof(double));
  for (uint32_t c = 1; c <= w; ++c) clog[c] = (double)c * log2((double)c);
  const double log_w = log2((double)w);
  const uint32_t nwin = n - w + 1;
  double* ent = (double*)malloc(sizeof(double) * nwin);
  uint32_t counts[32] = {0};
  double sum_clog = 0.0;
#define SYM(r) ((r) < 31 ? (r) : 31)
  for (uint32_t k = 0; k < w; ++k) {
    const unsigned s = SYM(seq[k]);
    sum_clog -= clog[counts[s]];
    counts[s] += 1;
    sum_clog += clog[counts[s]];
  }
  ent[0] = log_w - sum_clog / (double)w;
  for (uint32_t i = 1; i < nwin; ++i) {
    const unsigned out = SYM(seq[i - 1]);
    sum_clog -= clog[counts[out]];
    counts[out] -= 1;
    sum_clog += clog[counts[out]];
    const unsigned inn = SYM(seq[i + w - 1]);
    sum_clog -= clog[counts[inn]];
    counts[inn] += 1;
    sum_clog += clog[counts[inn]];
    ent[i] = log_w - sum_clog / (double)w;
  }
#undef SYM
  uint32_t i = 0;
  while (i < nwin) {
    if (ent[i] <= locut + 1e-12) {
      uint32_t lo = i, hi = i;
      while (lo > 0 && ent[lo - 1] <= hicut + 1e-12) --lo;
      while (hi + 1 < nwin && ent[hi + 1] <= hicut + 1e-12) ++hi;
      for (uint32_t k = lo; k < hi + w && k < n; ++k) mask[k] = 1;
      i = hi + 1;
    } else {
      ++i;
    }
  }
  free(clog);
  free(ent);
  uint32_t cnt = 0;
  for (uint32_t k = 0; k < n; ++k) cnt += mask[k];
  return cnt;
}
