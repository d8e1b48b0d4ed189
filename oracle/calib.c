/*
 * Per-profile calibration — TEST INFRASTRUCTURE ONLY.  A plain-C restatement of
 * the reference's calibrate_profile (src/evalue.rs:714-748):
 *
 *   * sample i draws from its own SplitMix64 stream, seeded by
 *     stream_seed(seed, 0xBEEF, i) (src/evalue.rs:53-81);
 *   * its length is lengths[below(n_lengths)], at least 1; its residues are
 *     i.i.d. from the BLOSUM62 background (BackgroundSampler, :84-114: the first
 *     cumulative probability above next_f64());
 *   * its score is the exact SW-Gotoh score of the profile rows against it;
 *   * a Gumbel is fitted by maximum likelihood (fit_gumbel_ml, :138-182: bisection
 *     of Lawless' equation; mu by gumbel_mu_given_lambda, :129-134), and
 *     K = exp(lambda (mu + 1/2)) / (m * mean length).
 *
 * Sums run in index order, as the reference's iterator sums do, so the fit is
 * the reference's to the last bit given the same libm.
 */
#include <math.h>
#include <stdlib.h>

#include "oracle.h"

#define GOLDEN 0x9E3779B97F4A7C15ull
#define OR_PI 3.141592653589793238462643383279502884 /* std::f64::consts::PI */

static uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* SplitMix64::next_u64: advance, then mix */
static uint64_t sm_next(uint64_t* s) {
  *s += GOLDEN;
  return mix64(*s);
}

static double sm_f64(uint64_t* s) { return (double)(sm_next(s) >> 11) / (double)(1ull << 53); }

uint64_t or_stream_seed(uint64_t seed, uint64_t c, uint64_t i) {
  uint64_t s = seed ^ (c * 0xA24BAED4963EE407ull) ^ (i * 0x9FB21C651E98DF25ull);
  return sm_next(&s);
}

void or_background_cum(const double* p_back20, double* cum20) {
  double total = 0.0;
  for (int i = 0; i < 20; ++i) total += p_back20[i];
  double acc = 0.0;
  for (int i = 0; i < 20; ++i) {
    acc += p_back20[i] / total;
    cum20[i] = acc;
  }
  cum20[19] = 1.0;
}

static uint8_t bg_sample(const double* cum, uint64_t* s) {
  const double u = sm_f64(s);
  for (int i = 0; i < 20; ++i)
    if (u < cum[i]) return (uint8_t)i;
  return 19;
}

uint32_t or_calibration_length(const uint32_t* lengths, uint32_t n_lengths, uint64_t seed, uint64_t i) {
  uint64_t s = or_stream_seed(seed, 0xBEEF, i);
  uint32_t n = lengths[sm_next(&s) % n_lengths];
  return n ? n : 1;
}

void or_calibration_target(const uint32_t* lengths, uint32_t n_lengths, uint64_t seed, uint64_t i, const double* cum20,
                           uint8_t* out, uint32_t* len) {
  uint64_t s = or_stream_seed(seed, 0xBEEF, i);
  uint32_t n = lengths[sm_next(&s) % n_lengths];
  if (n == 0) n = 1;
  for (uint32_t k = 0; k < n; ++k) out[k] = bg_sample(cum20, &s);
  *len = n;
}

/* src/evalue.rs:129-134 */
double or_gumbel_mu_given_lambda(const double* xs, uint64_t n, double lambda) {
  double xmin = INFINITY;
  for (uint64_t i = 0; i < n; ++i) xmin = fmin(xmin, xs[i]);
  double s = 0.0;
  for (uint64_t i = 0; i < n; ++i) s += exp(-lambda * (xs[i] - xmin));
  return xmin - log(s / (double)n) / lambda;
}

static double lawless_g(const double* xs, uint64_t n, double xmin, double mean, double lam) {
  double s0 = 0.0, s1 = 0.0;
  for (uint64_t i = 0; i < n; ++i) {
    const double w = exp(-lam * (xs[i] - xmin));
    s0 += w;
    s1 += xs[i] * w;
  }
  return 1.0 / lam - mean + s1 / s0;
}

/* src/evalue.rs:138-182; returns 0 where the reference returns None */
int or_fit_gumbel_ml(const double* xs, uint64_t n, double* lambda, double* mu) {
  if (n < 10) return 0;
  double sum = 0.0;
  for (uint64_t i = 0; i < n; ++i) sum += xs[i];
  const double mean = sum / (double)n;
  double ss = 0.0;
  for (uint64_t i = 0; i < n; ++i) ss += (xs[i] - mean) * (xs[i] - mean);
  const double var = ss / ((double)n - 1.0);
  if (isnan(var) || var <= 0.0) return 0;
  double xmin = INFINITY;
  for (uint64_t i = 0; i < n; ++i) xmin = fmin(xmin, xs[i]);
  const double lam0 = OR_PI / (sqrt(var) * sqrt(6.0));
  double lo = lam0 / 10.0, hi = lam0 * 10.0;
  if (lawless_g(xs, n, xmin, mean, lo) < 0.0 || lawless_g(xs, n, xmin, mean, hi) > 0.0) return 0;
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (lawless_g(xs, n, xmin, mean, mid) > 0.0)
      lo = mid;
    else
      hi = mid;
    if (hi - lo < 1e-12 * hi) break;
  }
  *lambda = 0.5 * (lo + hi);
  *mu = or_gumbel_mu_given_lambda(xs, n, *lambda);
  return 1;
}

int or_calibrate_profile(const int32_t* rows, uint32_t m, const uint32_t* lengths, uint32_t n_lengths,
                         uint32_t samples, uint64_t seed, const double* p_back20, int32_t open, int32_t ext,
                         int32_t* scores, double* lambda, double* k, double* mu, int nthreads) {
  if (n_lengths == 0 || m == 0) return 0;
  double cum[20];
  or_background_cum(p_back20, cum);
  uint32_t max_len = 1;
  for (uint32_t i = 0; i < n_lengths; ++i)
    if (lengths[i] > max_len) max_len = lengths[i];
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
  {
    uint8_t* t = (uint8_t*)malloc(max_len);
#pragma omp for schedule(dynamic, 16)
    for (int64_t i = 0; i < (int64_t)samples; ++i) {
      uint32_t n;
      or_calibration_target(lengths, n_lengths, seed, (uint64_t)i, cum, t, &n);
      scores[i] = or_gotoh_score(rows, m, t, n, open, ext);
    }
    free(t);
  }
  double* xs = (double*)malloc((samples ? samples : 1) * sizeof(double));
  for (uint32_t i = 0; i < samples; ++i) xs[i] = (double)scores[i];
  const int ok = or_fit_gumbel_ml(xs, samples, lambda, mu);
  free(xs);
  if (!ok) return 0;
  uint64_t lsum = 0;
  for (uint32_t i = 0; i < n_lengths; ++i) lsum += lengths[i];
  const double mean_len = (double)lsum / (double)n_lengths;
  *k = exp(*lambda * (*mu + 0.5)) / ((double)m * mean_len);
  return 1;
}
