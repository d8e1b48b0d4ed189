/*
 * CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle.h).  Plain C restatement of
 * the reference's exact scalar kernels.  Arithmetic is done in wrapping 32-bit
 * two's complement, which is what the reference's release build does on
 * overflow; no input used by the tests comes near it.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

#define NEG32 (INT32_MIN / 4) /* src/simd.rs:354, src/align.rs:287 */

static inline int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
static inline int32_t wsub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
static inline int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }
static inline int32_t score_of(const int32_t* row, uint8_t r) { return r < OR_NPROF ? row[r] : 0; }

/* src/ungapped.rs:38-46 */
void or_diag_range(uint64_t m, uint64_t n, int64_t d, uint64_t* lo, uint64_t* hi) {
  int64_t l = -d > 0 ? -d : 0;
  int64_t h = (int64_t)m < (int64_t)n - d ? (int64_t)m : (int64_t)n - d;
  if (h <= l) {
    *lo = 0;
    *hi = 0;
  } else {
    *lo = (uint64_t)l;
    *hi = (uint64_t)h;
  }
}

/* src/ungapped.rs:53-62 */
int32_t or_kadane_score(const int32_t* rows, const uint8_t* t, int64_t d, uint64_t lo, uint64_t hi) {
  int32_t best = 0, cur = 0;
  for (uint64_t q = lo; q < hi; ++q) {
    uint8_t tr = t[(int64_t)q + d];
    int32_t s = score_of(rows + q * OR_NPROF, tr);
    cur = wadd(imax(cur, 0), s);
    best = imax(best, cur);
  }
  return best;
}

/* src/ungapped.rs:69-88 */
int32_t or_kadane_segment(const int32_t* rows, const uint8_t* t, int64_t d, uint64_t lo, uint64_t hi,
                          uint64_t* q_start, uint64_t* q_end) {
  int32_t best = 0, cur = 0;
  uint64_t bs = 0, be = 0, cs = lo;
  for (uint64_t q = lo; q < hi; ++q) {
    uint8_t tr = t[(int64_t)q + d];
    int32_t s = score_of(rows + q * OR_NPROF, tr);
    if (cur <= 0) {
      cur = s;
      cs = q;
    } else {
      cur = wadd(cur, s);
    }
    if (cur > best) {
      best = cur;
      bs = cs;
      be = q;
    }
  }
  *q_start = bs;
  *q_end = be;
  return best;
}

/* src/simd.rs:347-390 (scalar_gotoh_score_end) */
int or_gotoh_score_end(const int32_t* rows, uint32_t m, const uint8_t* t, uint32_t n, int32_t open,
                       int32_t ext, int32_t* score, uint32_t* qi, uint32_t* tj) {
  int32_t* h_prev = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
  int32_t* h_cur = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
  int32_t* f_col = (int32_t*)malloc(((size_t)n + 1) * sizeof(int32_t));
  for (uint32_t j = 0; j <= n; ++j) f_col[j] = NEG32;
  int32_t best = 0;
  uint32_t bi = 0;
  uint64_t bj = UINT64_MAX;
  for (uint32_t i = 0; i < m; ++i) {
    const int32_t* row = rows + (size_t)i * OR_NPROF;
    int32_t e = NEG32;
    h_cur[0] = 0;
    for (uint32_t j = 1; j <= n; ++j) {
      int32_t sc = score_of(row, t[j - 1]);
      int32_t diag = wadd(h_prev[j - 1], sc);
      e = imax(wsub(h_cur[j - 1], open), wsub(e, ext));
      int32_t f = imax(wsub(h_prev[j], open), wsub(f_col[j], ext));
      f_col[j] = f;
      int32_t v = imax(imax(imax(diag, e), f), 0);
      h_cur[j] = v;
      if (v > best || (v == best && v > 0 && (uint64_t)(j - 1) < bj)) {
        best = v;
        bi = i;
        bj = j - 1;
      }
    }
    int32_t* tmp = h_prev;
    h_prev = h_cur;
    h_cur = tmp;
  }
  free(h_prev);
  free(h_cur);
  free(f_col);
  if (best > 0) {
    *score = best;
    *qi = bi;
    *tj = (uint32_t)bj;
    return 1;
  }
  *score = 0;
  *qi = 0;
  *tj = 0;
  return 0;
}

/* src/simd.rs:252-255 (empty inputs) and 342-345 (score only) */
int32_t or_gotoh_score(const int32_t* rows, uint32_t m, const uint8_t* t, uint32_t n, int32_t open,
                       int32_t ext) {
  if (m == 0 || n == 0) return 0;
  int32_t s;
  uint32_t a, b;
  or_gotoh_score_end(rows, m, t, n, open, ext, &s, &a, &b);
  return s;
}

/* src/simd.rs:1124-1142: independent three-matrix Gotoh (small cases only: O(m*n) memory) */
int32_t or_reference_score(const int32_t* rows, uint32_t m, const uint8_t* t, uint32_t n, int32_t open,
                           int32_t ext) {
  size_t w = (size_t)n + 1;
  int32_t* h = (int32_t*)calloc(((size_t)m + 1) * w, sizeof(int32_t));
  int32_t* e = (int32_t*)malloc(((size_t)m + 1) * w * sizeof(int32_t));
  int32_t* f = (int32_t*)malloc(((size_t)m + 1) * w * sizeof(int32_t));
  for (size_t k = 0; k < ((size_t)m + 1) * w; ++k) e[k] = f[k] = NEG32;
  int32_t best = 0;
  for (uint32_t i = 1; i <= m; ++i) {
    for (uint32_t j = 1; j <= n; ++j) {
      size_t c = (size_t)i * w + j;
      e[c] = imax(wsub(h[c - 1], open), wsub(e[c - 1], ext));
      f[c] = imax(wsub(h[c - w], open), wsub(f[c - w], ext));
      int32_t sc = score_of(rows + (size_t)(i - 1) * OR_NPROF, t[j - 1]);
      h[c] = imax(imax(imax(wadd(h[c - w - 1], sc), e[c]), f[c]), 0);
      best = imax(best, h[c]);
    }
  }
  free(h);
  free(e);
  free(f);
  return best;
}

/* src/align.rs:408-493, score part of local_full_tb with band = Some((center, radius));
 * radius < 0 means no band.  Returns 0 when no positive alignment exists (None). */
int32_t or_band_score(const int32_t* rows, uint32_t m, const uint8_t* t, uint32_t n, int32_t open,
                      int32_t ext, int64_t center, int64_t radius) {
  if (m == 0 || n == 0) return 0;
  int32_t* h_prev = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
  int32_t* h_cur = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
  int32_t* f_col = (int32_t*)malloc(((size_t)n + 1) * sizeof(int32_t));
  for (uint32_t j = 0; j <= n; ++j) f_col[j] = NEG32;
  int32_t best = 0;
  for (uint32_t i = 1; i <= m; ++i) {
    const int32_t* row = rows + (size_t)(i - 1) * OR_NPROF;
    int32_t e = NEG32;
    h_cur[0] = 0;
    for (uint32_t j = 1; j <= n; ++j) {
      if (radius >= 0) {
        int64_t off = (int64_t)j - (int64_t)i - center;
        if (off < 0) off = -off;
        if (off > radius) {
          h_cur[j] = 0;
          f_col[j] = NEG32;
          e = NEG32;
          continue;
        }
      }
      int32_t diag = wadd(h_prev[j - 1], score_of(row, t[j - 1]));
      int32_t e_open = wsub(h_cur[j - 1], open);
      int32_t e_ext = wsub(e, ext);
      e = e_ext > e_open ? e_ext : e_open;
      int32_t f_open = wsub(h_prev[j], open);
      int32_t f_ext = wsub(f_col[j], ext);
      int32_t f = f_ext > f_open ? f_ext : f_open;
      f_col[j] = f;
      int32_t v = diag;
      if (e > v) v = e;
      if (f > v) v = f;
      if (v <= 0) v = 0;
      h_cur[j] = v;
      if (v > best) best = v;
    }
    int32_t* tmp = h_prev;
    h_prev = h_cur;
    h_cur = tmp;
  }
  free(h_prev);
  free(h_cur);
  free(f_col);
  return best;
}

void or_sw_pairs(const int32_t* rows_arena, const uint64_t* row_off, const uint32_t* qlen,
                 const uint8_t* tgt_arena, const uint64_t* tgt_off, const uint32_t* pq, const uint32_t* pt,
                 const int64_t* center, const int64_t* radius, uint64_t n_pairs, int32_t open, int32_t ext,
                 int32_t* out, int nthreads) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1)
  for (int64_t k = 0; k < (int64_t)n_pairs; ++k) {
    uint32_t q = pq[k], tt = pt[k];
    const int32_t* rows = rows_arena + row_off[q] * OR_NPROF;
    const uint8_t* t = tgt_arena + tgt_off[tt];
    uint32_t n = (uint32_t)(tgt_off[tt + 1] - tgt_off[tt]);
    if (radius && radius[k] >= 0)
      out[k] = or_band_score(rows, qlen[q], t, n, open, ext, center[k], radius[k]);
    else
      out[k] = or_gotoh_score(rows, qlen[q], t, n, open, ext);
  }
}

void or_ungapped_hits(const int32_t* rows_arena, const uint64_t* row_off, const uint32_t* qlen,
                      const uint8_t* tgt_arena, const uint64_t* tgt_off, const uint32_t* hq, const uint32_t* ht,
                      const int32_t* hd, uint64_t n_hits, int32_t* out, int nthreads) {
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads > 0 ? nthreads : 1)
  for (int64_t k = 0; k < (int64_t)n_hits; ++k) {
    uint32_t q = hq[k], tt = ht[k];
    const int32_t* rows = rows_arena + row_off[q] * OR_NPROF;
    const uint8_t* t = tgt_arena + tgt_off[tt];
    uint64_t n = tgt_off[tt + 1] - tgt_off[tt], lo, hi;
    or_diag_range(qlen[q], n, hd[k], &lo, &hi);
    out[k] = or_kadane_score(rows, t, hd[k], lo, hi);
  }
}
