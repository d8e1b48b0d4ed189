/*
 * CPU baseline for ungapped diagonal scoring — TEST/BENCH INFRASTRUCTURE ONLY.
 * A C restatement of the reference's own CPU path for seed-hit diagonals on
 * AVX2 (the kernel the reference picks by default on x86-64):
 *
 *   * the biased u8 diagonal profile, one 32-entry table per query position,
 *     bias = -min score, limit = 255 - (max + bias); a profile with bias > 255
 *     or limit < 64 is not used and every lane is scored by the scalar Kadane
 *     (DiagProfile::rebuild, src/ungapped.rs:209-250);
 *   * the jobs of one query ordered by window start (counting sort) so that a
 *     batch of 32 lanes covers the same query positions (score_and_gate,
 *     src/prefilter.rs:1529-1548);
 *   * per batch: the lanes' residues copied lane-major over the 16-aligned union
 *     window (sentinel outside each lane's window), transposed in 16 x 16 byte
 *     blocks to position-major, then the saturating u8 Kadane over the union
 *     window with two 16-byte table lookups per position
 *     (score_batch / kadane_avx2, src/ungapped.rs:285-386, 437-456);
 *   * lanes whose u8 best exceeds the limit rescored exactly (scalar Kadane).
 *
 * Queries in parallel over all host threads. bench.py times it as the CPU
 * baseline of row (U); its results are checked against the scalar oracle.
 */
#include <immintrin.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define NPROF 21
#define SENT 21
#define LANES 32
#define MIN_LIMIT 64

/* 16 x 16 byte block transpose: row r (16 bytes at src + r*ss) becomes column r
 * of the output (16 rows at dst + c*ds); every byte clamped to the sentinel. */
static void transpose16(const uint8_t* src, size_t ss, uint8_t* dst, size_t ds) {
  const __m128i cap = _mm_set1_epi8((char)SENT);
  __m128i a[16], b[16], c[16], e[16];
  for (int r = 0; r < 16; ++r) a[r] = _mm_min_epu8(_mm_loadu_si128((const __m128i*)(src + r * ss)), cap);
  for (int k = 0; k < 8; ++k) {
    b[2 * k] = _mm_unpacklo_epi8(a[2 * k], a[2 * k + 1]);
    b[2 * k + 1] = _mm_unpackhi_epi8(a[2 * k], a[2 * k + 1]);
  }
  for (int j = 0; j < 4; ++j) {
    c[4 * j] = _mm_unpacklo_epi16(b[4 * j], b[4 * j + 2]);
    c[4 * j + 1] = _mm_unpackhi_epi16(b[4 * j], b[4 * j + 2]);
    c[4 * j + 2] = _mm_unpacklo_epi16(b[4 * j + 1], b[4 * j + 3]);
    c[4 * j + 3] = _mm_unpackhi_epi16(b[4 * j + 1], b[4 * j + 3]);
  }
  for (int i = 0; i < 2; ++i)
    for (int q = 0; q < 4; ++q) {
      e[8 * i + 2 * q] = _mm_unpacklo_epi32(c[8 * i + q], c[8 * i + 4 + q]);
      e[8 * i + 2 * q + 1] = _mm_unpackhi_epi32(c[8 * i + q], c[8 * i + 4 + q]);
    }
  for (int k = 0; k < 8; ++k) {
    _mm_storeu_si128((__m128i*)(dst + (2 * k) * ds), _mm_unpacklo_epi64(e[k], e[8 + k]));
    _mm_storeu_si128((__m128i*)(dst + (2 * k + 1) * ds), _mm_unpackhi_epi64(e[k], e[8 + k]));
  }
}

typedef struct {
  uint32_t lo, hi;  /* query window */
  int64_t diag;
  const uint8_t* t; /* target residues */
  uint32_t job;     /* output index */
} lane_job;

static void score_query(const int32_t* rows, uint32_t m, const uint8_t* tables, int simd, uint8_t bias, uint8_t limit,
                        lane_job* jobs, uint32_t nj, int32_t* out, uint8_t* lm, uint8_t* pm, uint32_t* cnt,
                        lane_job* ord) {
  /* counting sort of the jobs by window start */
  memset(cnt, 0, (m + 2) * sizeof(uint32_t));
  for (uint32_t j = 0; j < nj; ++j) cnt[jobs[j].lo + 1]++;
  for (uint32_t q = 0; q <= m; ++q) cnt[q + 1] += cnt[q];
  for (uint32_t j = 0; j < nj; ++j) ord[cnt[jobs[j].lo]++] = jobs[j];
  for (uint32_t c0 = 0; c0 < nj; c0 += LANES) {
    const uint32_t c1 = c0 + LANES < nj ? c0 + LANES : nj;
    if (!simd) {
      for (uint32_t k = c0; k < c1; ++k)
        out[ord[k].job] = or_kadane_score(rows, ord[k].t, ord[k].diag, ord[k].lo, ord[k].hi);
      continue;
    }
    uint32_t q_lo = m, q_hi = 0;
    for (uint32_t k = c0; k < c1; ++k)
      if (ord[k].lo < ord[k].hi) {
        if (ord[k].lo < q_lo) q_lo = ord[k].lo;
        if (ord[k].hi > q_hi) q_hi = ord[k].hi;
      }
    uint8_t best[LANES];
    memset(best, 0, sizeof best);
    if (q_lo < q_hi) {
      const uint32_t a = q_lo & ~15u, b = (q_hi + 15) & ~15u, w = b - a;
      /* lane-major copy of each lane's diagonal, sentinel outside its window */
      for (uint32_t l = 0; l < LANES; ++l) {
        uint8_t* row = lm + (size_t)l * w;
        memset(row, SENT, w);
        const uint32_t k = c0 + l;
        if (k >= c1 || ord[k].lo >= ord[k].hi) continue;
        memcpy(row + (ord[k].lo - a), ord[k].t + (int64_t)ord[k].lo + ord[k].diag, ord[k].hi - ord[k].lo);
      }
      /* 16 x 16 transposes to position-major pm[i * LANES + lane] */
      for (uint32_t g = 0; g < LANES / 16; ++g)
        for (uint32_t pb = 0; pb < w / 16; ++pb)
          transpose16(lm + (size_t)(g * 16) * w + pb * 16, w, pm + (size_t)(pb * 16) * LANES + g * 16, LANES);
      /* saturating u8 Kadane over the union window */
      const __m256i vbias = _mm256_set1_epi8((char)bias), v15 = _mm256_set1_epi8(15);
      __m256i cur = _mm256_setzero_si256(), bst = _mm256_setzero_si256();
      for (uint32_t i = q_lo; i < q_hi; ++i) {
        const __m256i t = _mm256_loadu_si256((const __m256i*)(pm + (size_t)(i - a) * LANES));
        const __m256i lo = _mm256_broadcastsi128_si256(_mm_loadu_si128((const __m128i*)(tables + (size_t)i * 32)));
        const __m256i hi =
            _mm256_broadcastsi128_si256(_mm_loadu_si128((const __m128i*)(tables + (size_t)i * 32 + 16)));
        const __m256i sc = _mm256_blendv_epi8(_mm256_shuffle_epi8(lo, t), _mm256_shuffle_epi8(hi, t),
                                              _mm256_cmpgt_epi8(t, v15));
        cur = _mm256_subs_epu8(_mm256_adds_epu8(cur, sc), vbias);
        bst = _mm256_max_epu8(bst, cur);
      }
      _mm256_storeu_si256((__m256i*)best, bst);
    }
    for (uint32_t k = c0; k < c1; ++k) {
      const uint8_t bv = best[k - c0];
      out[ord[k].job] = bv > limit ? or_kadane_score(rows, ord[k].t, ord[k].diag, ord[k].lo, ord[k].hi) : (int32_t)bv;
    }
  }
}

void or_ungapped_hits_avx2(const int32_t* rows_arena, const uint64_t* row_off, const uint32_t* qlen,
                           const uint8_t* tgt_arena, const uint64_t* tgt_off, const uint32_t* hq, const uint32_t* ht,
                           const int32_t* hd, uint64_t n_hits, int32_t* out, int nthreads) {
  /* runs of hits with the same query (hits arrive grouped by query) */
  uint64_t n_runs = 0;
  for (uint64_t k = 0; k < n_hits; ++k)
    if (k == 0 || hq[k] != hq[k - 1]) ++n_runs;
  uint64_t* run = (uint64_t*)malloc((n_runs + 1) * sizeof(uint64_t));
  uint64_t r = 0;
  for (uint64_t k = 0; k < n_hits; ++k)
    if (k == 0 || hq[k] != hq[k - 1]) run[r++] = k;
  run[n_runs] = n_hits;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
  {
    size_t cap_m = 0, cap_j = 0, cap_w = 0;
    uint8_t *tables = NULL, *lm = NULL, *pm = NULL;
    uint32_t* cnt = NULL;
    lane_job *jobs = NULL, *ord = NULL;
#pragma omp for schedule(dynamic, 1)
    for (int64_t ri = 0; ri < (int64_t)n_runs; ++ri) {
      const uint64_t k0 = run[ri], k1 = run[ri + 1];
      const uint32_t q = hq[k0];
      const int32_t* rows = rows_arena + row_off[q] * NPROF;
      const uint32_t m = qlen[q];
      /* the biased u8 tables (codes 21..31 score 0) */
      int32_t lo = 0, hi = 0;
      for (size_t i = 0; i < (size_t)m * NPROF; ++i) {
        if (rows[i] < lo) lo = rows[i];
        if (rows[i] > hi) hi = rows[i];
      }
      const int32_t bias = -lo, limit = 255 - (hi + bias);
      const int simd = m > 0 && bias <= 255 && limit >= MIN_LIMIT;
      if (m + 2 > cap_m) {
        cap_m = m + 2;
        free(tables);
        free(cnt);
        tables = (uint8_t*)malloc(cap_m * 32);
        cnt = (uint32_t*)malloc((cap_m + 2) * sizeof(uint32_t));
      }
      if (simd)
        for (uint32_t i = 0; i < m; ++i) {
          for (int res = 0; res < 32; ++res) tables[(size_t)i * 32 + res] = (uint8_t)bias;
          for (int res = 0; res < NPROF; ++res) tables[(size_t)i * 32 + res] = (uint8_t)(rows[(size_t)i * NPROF + res] + bias);
        }
      const uint32_t nj = (uint32_t)(k1 - k0);
      if (nj > cap_j) {
        cap_j = nj;
        free(jobs);
        free(ord);
        jobs = (lane_job*)malloc(cap_j * sizeof(lane_job));
        ord = (lane_job*)malloc(cap_j * sizeof(lane_job));
      }
      const size_t wmax = ((size_t)m + 31) & ~(size_t)15;
      if (wmax * LANES > cap_w) {
        cap_w = wmax * LANES;
        free(lm);
        free(pm);
        lm = (uint8_t*)malloc(cap_w + 64);
        pm = (uint8_t*)malloc(cap_w + 64);
      }
      for (uint32_t j = 0; j < nj; ++j) {
        const uint64_t k = k0 + j;
        const uint64_t tn = tgt_off[ht[k] + 1] - tgt_off[ht[k]];
        uint64_t a, b;
        or_diag_range(m, tn, hd[k], &a, &b);
        jobs[j] = (lane_job){(uint32_t)a, (uint32_t)b, hd[k], tgt_arena + tgt_off[ht[k]], (uint32_t)k};
      }
      score_query(rows, m, tables, simd, (uint8_t)(simd ? bias : 0), (uint8_t)(simd ? limit : 0), jobs, nj, out,
                  lm, pm, cnt, ord);
    }
    free(tables);
    free(cnt);
    free(jobs);
    free(ord);
    free(lm);
    free(pm);
  }
  free(run);
}

/* One query's jobs with explicit windows (the reference's score_batch calls from
 * score_and_gate, src/prefilter.rs:1529-1575): tp[j] = target residues,
 * window [lo[j], hi[j]) on diagonal d[j]; out[j] = kadane_score. */
void or_kadane_jobs_avx2(const int32_t* rows, uint32_t m, const uint8_t* const* tp, const int64_t* d,
                         const uint32_t* lo, const uint32_t* hi, uint32_t n, int32_t* out) {
  if (n == 0) return;
  int32_t mn = 0, mx = 0;
  for (size_t i = 0; i < (size_t)m * NPROF; ++i) {
    if (rows[i] < mn) mn = rows[i];
    if (rows[i] > mx) mx = rows[i];
  }
  const int32_t bias = -mn, limit = 255 - (mx + bias);
  const int simd = m > 0 && bias <= 255 && limit >= MIN_LIMIT;
  uint8_t* tables = (uint8_t*)malloc(((size_t)m + 2) * 32);
  if (simd)
    for (uint32_t i = 0; i < m; ++i) {
      for (int res = 0; res < 32; ++res) tables[(size_t)i * 32 + res] = (uint8_t)bias;
      for (int res = 0; res < NPROF; ++res) tables[(size_t)i * 32 + res] = (uint8_t)(rows[(size_t)i * NPROF + res] + bias);
    }
  uint32_t* cnt = (uint32_t*)malloc(((size_t)m + 4) * sizeof(uint32_t));
  lane_job* jobs = (lane_job*)malloc((size_t)n * sizeof(lane_job));
  lane_job* ord = (lane_job*)malloc((size_t)n * sizeof(lane_job));
  const size_t wmax = ((size_t)m + 31) & ~(size_t)15;
  uint8_t* lm = (uint8_t*)malloc(wmax * LANES + 64);
  uint8_t* pm = (uint8_t*)malloc(wmax * LANES + 64);
  for (uint32_t j = 0; j < n; ++j) jobs[j] = (lane_job){lo[j], hi[j] > lo[j] ? hi[j] : lo[j], d[j], tp[j], j};
  score_query(rows, m, tables, simd, (uint8_t)(simd ? bias : 0), (uint8_t)(simd ? limit : 0), jobs, n, out, lm, pm, cnt,
              ord);
  free(tables);
  free(cnt);
  free(jobs);
  free(ord);
  free(lm);
  free(pm);
}
