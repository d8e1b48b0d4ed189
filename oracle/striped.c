/*
 * CPU baseline — TEST/BENCH INFRASTRUCTURE ONLY.  A C restatement of the
 * reference's own CPU scoring path for QueryProfile::sw_score_with
 * (src/simd.rs:252-292) on AVX2, the kernel family the reference picks by
 * default on x86-64 (src/simd.rs:99-124):
 *
 *   1. biased u8 Farrar striped pass, 32 lanes, with lazy-F and the headroom
 *      test (StripedU8 src/simd.rs:418-472, kernel macro :516-592);
 *   2. on headroom exceeded, the i16 striped pass, 16 lanes, lazy-F, saturation
 *      test (Striped src/simd.rs:715-754, kernels :813-897);
 *   3. on saturation, open <= extend or rows outside i16: the exact scalar
 *      Gotoh (src/simd.rs:342-390, or_gotoh_score).
 *
 * Query profiles are built once per query and its targets scored in turn,
 * queries in parallel over all host threads (rayon's per-query map in
 * Engine::search_batch, src/search.rs:708-730).  Used by bench.py as the timed
 * CPU baseline; scores are checked against the scalar oracle by the tests.
 */
#include <immintrin.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define NPROF 21
#define MIN_U8_LIMIT 96 /* src/simd.rs:432 */

typedef struct {
  int seg_len;
  uint8_t bias, limit;
  __m256i* data; /* (NPROF + 1) * seg_len vectors */
} prof_u8;

typedef struct {
  int seg_len;
  __m256i* data;
} prof_i16;

static void* amalloc(size_t n) {
  void* p = NULL;
  if (posix_memalign(&p, 64, n ? n : 64)) return NULL;
  return p;
}

/* StripedU8::build, src/simd.rs:435-472; returns 0 when not built */
static int build_u8(const int32_t* rows, int m, prof_u8* p) {
  const int L = 32;
  if (m == 0) return 0;
  int lo = 0, hi = 0;
  for (int i = 0; i < m * NPROF; ++i) {
    if (rows[i] < lo) lo = rows[i];
    if (rows[i] > hi) hi = rows[i];
  }
  int bias = -lo, limit = 255 - (hi + bias);
  if (bias > 255 || limit < MIN_U8_LIMIT) return 0;
  int seg = (m + L - 1) / L;
  p->seg_len = seg;
  p->bias = (uint8_t)bias;
  p->limit = (uint8_t)limit;
  p->data = (__m256i*)amalloc((size_t)(NPROF + 1) * seg * 32);
  uint8_t* d = (uint8_t*)p->data;
  for (int res = 0; res <= NPROF; ++res)
    for (int i = 0; i < seg; ++i)
      for (int l = 0; l < L; ++l) {
        int col = i + l * seg;
        int v = (col < m && res < NPROF) ? rows[col * NPROF + res] : 0;
        d[(size_t)(res * seg + i) * L + l] = (uint8_t)(v + bias);
      }
  return 1;
}

/* Striped::build, src/simd.rs:730-754 */
static int build_i16(const int32_t* rows, int m, prof_i16* p) {
  const int L = 16;
  if (m == 0) return 0;
  int seg = (m + L - 1) / L;
  for (int i = 0; i < m * NPROF; ++i)
    if (rows[i] > 32767 || rows[i] < -32768) return 0;
  p->seg_len = seg;
  p->data = (__m256i*)amalloc((size_t)(NPROF + 1) * seg * 32);
  int16_t* d = (int16_t*)p->data;
  for (int res = 0; res <= NPROF; ++res)
    for (int i = 0; i < seg; ++i)
      for (int l = 0; l < L; ++l) {
        int col = i + l * seg;
        int v = (col < m && res < NPROF) ? rows[col * NPROF + res] : 0;
        d[(size_t)(res * seg + i) * L + l] = (int16_t)v;
      }
  return 1;
}

static inline __m256i shl1_u8(__m256i v) { return _mm256_alignr_epi8(v, _mm256_permute2x128_si256(v, v, 0x08), 15); }
static inline __m256i shl1_i16(__m256i v) { return _mm256_alignr_epi8(v, _mm256_permute2x128_si256(v, v, 0x08), 14); }

static inline int hmax_u8(__m256i v) {
  __m128i m = _mm_max_epu8(_mm256_castsi256_si128(v), _mm256_extracti128_si256(v, 1));
  m = _mm_max_epu8(m, _mm_srli_si128(m, 8));
  m = _mm_max_epu8(m, _mm_srli_si128(m, 4));
  m = _mm_max_epu8(m, _mm_srli_si128(m, 2));
  m = _mm_max_epu8(m, _mm_srli_si128(m, 1));
  return _mm_cvtsi128_si32(m) & 0xFF;
}

static inline int hmax_i16(__m256i v) {
  __m128i m = _mm_max_epi16(_mm256_castsi256_si128(v), _mm256_extracti128_si256(v, 1));
  m = _mm_max_epi16(m, _mm_shuffle_epi32(m, 0x4E));
  m = _mm_max_epi16(m, _mm_shuffle_epi32(m, 0x01));
  m = _mm_max_epi16(m, _mm_shufflelo_epi16(m, 0x01));
  return (int16_t)_mm_extract_epi16(m, 0);
}

typedef struct {
  __m256i *hs, *hl, *ea;
  int cap;
} scratch;

static void scratch_fit(scratch* s, int seg) {
  if (s->cap >= seg) return;
  free(s->hs);
  free(s->hl);
  free(s->ea);
  s->hs = (__m256i*)amalloc((size_t)seg * 32);
  s->hl = (__m256i*)amalloc((size_t)seg * 32);
  s->ea = (__m256i*)amalloc((size_t)seg * 32);
  s->cap = seg;
}

/* striped_u8_kernel!, src/simd.rs:516-592: -1 when the headroom was exceeded */
static int score_u8(const prof_u8* p, const uint8_t* t, int n, int open, int ext, scratch* s) {
  const int seg = p->seg_len;
  scratch_fit(s, seg);
  const __m256i vopen = _mm256_set1_epi8((char)(uint8_t)open), vext = _mm256_set1_epi8((char)(uint8_t)ext);
  const __m256i vbias = _mm256_set1_epi8((char)p->bias), vzero = _mm256_setzero_si256();
  const __m256i vlimit = _mm256_set1_epi8((char)p->limit);
  __m256i *hs = s->hs, *hl = s->hl, *ea = s->ea;
  for (int i = 0; i < seg; ++i) hs[i] = hl[i] = ea[i] = vzero;
  __m256i vmax = vzero;
  for (int j = 0; j < n; ++j) {
    const int r = t[j] < NPROF ? t[j] : NPROF;
    const __m256i* prof = p->data + (size_t)r * seg;
    __m256i vh = shl1_u8(hs[seg - 1]);
    __m256i vf = vzero;
    __m256i* tmp = hs;
    hs = hl;
    hl = tmp;
    for (int i = 0; i < seg; ++i) {
      const __m256i e = ea[i];
      vh = _mm256_subs_epu8(_mm256_adds_epu8(vh, _mm256_load_si256(prof + i)), vbias);
      vh = _mm256_max_epu8(vh, e);
      vh = _mm256_max_epu8(vh, vf);
      vmax = _mm256_max_epu8(vmax, vh);
      hs[i] = vh;
      const __m256i vho = _mm256_subs_epu8(vh, vopen);
      ea[i] = _mm256_max_epu8(_mm256_subs_epu8(e, vext), vho);
      vf = _mm256_max_epu8(_mm256_subs_epu8(vf, vext), vho);
      vh = hl[i];
    }
    for (int k = 0; k < 32; ++k) {
      vf = shl1_u8(vf);
      int done = 0;
      for (int i = 0; i < seg; ++i) {
        const __m256i h = _mm256_max_epu8(hs[i], vf);
        vmax = _mm256_max_epu8(vmax, h);
        hs[i] = h;
        const __m256i vho = _mm256_subs_epu8(h, vopen);
        ea[i] = _mm256_max_epu8(ea[i], vho);
        vf = _mm256_subs_epu8(vf, vext);
        if ((uint32_t)_mm256_movemask_epi8(_mm256_cmpeq_epi8(_mm256_subs_epu8(vf, vho), vzero)) == 0xFFFFFFFFu) {
          done = 1;
          break;
        }
      }
      if (done) break;
    }
    if ((uint32_t)_mm256_movemask_epi8(_mm256_cmpeq_epi8(_mm256_subs_epu8(vmax, vlimit), vzero)) != 0xFFFFFFFFu)
      return -1;
  }
  s->hs = hs;
  s->hl = hl;
  return hmax_u8(vmax);
}

/* striped_kernels! score, src/simd.rs:827-897: -1 when saturated */
static int score_i16(const prof_i16* p, const uint8_t* t, int n, int open, int ext, scratch* s) {
  const int seg = p->seg_len;
  scratch_fit(s, seg);
  const __m256i vopen = _mm256_set1_epi16((short)open), vext = _mm256_set1_epi16((short)ext);
  const __m256i vzero = _mm256_setzero_si256(), vneg = _mm256_set1_epi16(-32768);
  const __m256i lane0 = _mm256_set_epi16(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -32768);
  const __m256i sat = _mm256_set1_epi16(32767);
  __m256i *hs = s->hs, *hl = s->hl, *ea = s->ea;
  for (int i = 0; i < seg; ++i) hs[i] = hl[i] = ea[i] = vzero;
  __m256i vmax = vzero;
  for (int j = 0; j < n; ++j) {
    const int r = t[j] < NPROF ? t[j] : NPROF;
    const __m256i* prof = p->data + (size_t)r * seg;
    __m256i vh = shl1_i16(hs[seg - 1]);
    __m256i vf = vneg;
    __m256i* tmp = hs;
    hs = hl;
    hl = tmp;
    for (int i = 0; i < seg; ++i) {
      const __m256i e = ea[i];
      vh = _mm256_adds_epi16(vh, _mm256_load_si256(prof + i));
      vh = _mm256_max_epi16(vh, e);
      vh = _mm256_max_epi16(vh, vf);
      vh = _mm256_max_epi16(vh, vzero);
      vmax = _mm256_max_epi16(vmax, vh);
      hs[i] = vh;
      const __m256i vho = _mm256_subs_epi16(vh, vopen);
      ea[i] = _mm256_max_epi16(_mm256_subs_epi16(e, vext), vho);
      vf = _mm256_max_epi16(_mm256_subs_epi16(vf, vext), vho);
      vh = hl[i];
    }
    for (int k = 0; k < 16; ++k) {
      vf = _mm256_or_si256(shl1_i16(vf), lane0);
      int done = 0;
      for (int i = 0; i < seg; ++i) {
        const __m256i h = _mm256_max_epi16(hs[i], vf);
        vmax = _mm256_max_epi16(vmax, h);
        hs[i] = h;
        const __m256i vho = _mm256_subs_epi16(h, vopen);
        ea[i] = _mm256_max_epi16(ea[i], vho);
        vf = _mm256_subs_epi16(vf, vext);
        if (_mm256_movemask_epi8(_mm256_cmpgt_epi16(vf, vho)) == 0) {
          done = 1;
          break;
        }
      }
      if (done) break;
    }
  }
  s->hs = hs;
  s->hl = hl;
  if (_mm256_movemask_epi8(_mm256_cmpeq_epi16(vmax, sat)) != 0) return -1;
  return hmax_i16(vmax);
}

/* One query's targets; kernel_used[k]: 1 = u8, 2 = i16, 3 = scalar, 0 = empty */
static void score_query(const int32_t* rows, int m, const uint8_t* tgt_arena, const uint64_t* tgt_off,
                        const uint32_t* tlist, uint64_t nt, int open, int ext, int32_t* out, uint8_t* used,
                        scratch* s) {
  prof_u8 pu = {0};
  prof_i16 pi = {0};
  const int simd_ok = open > ext && open <= 32767 && ext >= 0; /* src/simd.rs:240-242 */
  const int have_u8 = simd_ok && build_u8(rows, m, &pu);
  const int have_i16 = simd_ok && build_i16(rows, m, &pi);
  for (uint64_t k = 0; k < nt; ++k) {
    const uint8_t* t = tgt_arena + tgt_off[tlist[k]];
    const int n = (int)(tgt_off[tlist[k] + 1] - tgt_off[tlist[k]]);
    int r = -1, kind = 0;
    if (m == 0 || n == 0) {
      r = 0;
    } else {
      if (have_u8 && open <= 255) {
        r = score_u8(&pu, t, n, open, ext, s);
        kind = 1;
      }
      if (r < 0 && have_i16) {
        r = score_i16(&pi, t, n, open, ext, s);
        kind = 2;
      }
      if (r < 0) {
        r = or_gotoh_score(rows, (uint32_t)m, t, (uint32_t)n, open, ext);
        kind = 3;
      }
    }
    out[k] = r;
    if (used) used[k] = (uint8_t)kind;
  }
  free(pu.data);
  free(pi.data);
}

/* Pairs grouped by query: query q's targets are tlist[qstart[q] .. qstart[q+1]). */
void or_striped_queries(const int32_t* rows_arena, const uint64_t* row_off, const uint32_t* qlen, uint32_t n_queries,
                        const uint8_t* tgt_arena, const uint64_t* tgt_off, const uint64_t* qstart,
                        const uint32_t* tlist, int32_t open, int32_t ext, int32_t* out, uint8_t* used,
                        int nthreads) {
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
  {
    scratch s = {0};
#pragma omp for schedule(dynamic, 1)
    for (int64_t q = 0; q < (int64_t)n_queries; ++q) {
      const uint64_t a = qstart[q], b = qstart[q + 1];
      if (a == b) continue;
      score_query(rows_arena + row_off[q] * NPROF, (int)qlen[q], tgt_arena, tgt_off, tlist + a, b - a, open, ext,
                  out + a, used ? used + a : NULL, &s);
    }
    free(s.hs);
    free(s.hl);
    free(s.ea);
  }
}
