/*
 * Prefilter evidence, chaining and gate — TEST/BENCH INFRASTRUCTURE ONLY.
 * A plain-C restatement of the reference's segment-evidence stage for one
 * query's seed hits (xdrop = 0, the default):
 *
 *   * hits grouped by target, then by diagonal (the packed-key radix sort,
 *     src/prefilter.rs:1021-1054); targets with fewer than min_hits hits are
 *     dropped (:1438-1440);
 *   * the max_diagonals diagonals with the most hits, ties to the smaller
 *     diagonal (top_diagonals, :1194-1225); dropped when the best has fewer
 *     than diag_hits hits (:1455-1457);
 *   * one job per kept diagonal (at most 16), window [qmin - diag_window,
 *     qmax + span + diag_window) clipped to diag_range, or the whole diagonal
 *     when diag_window = 0 (:1459-1474);
 *   * each job's best ungapped segment (kadane_score, src/ungapped.rs:53-62,
 *     batched as score_batch; positions by kadane_segment, :69-88);
 *   * the best single segment (first maximum in job order) or the best chain
 *     of two co-linear segments x -> y, sx + sy - gap(|dy - dx|), accepted when
 *     qe_x < qs_y and qe_x + dx < qs_y + dy (score_and_gate, src/prefilter.rs:
 *     1577-1637; GapCosts::cost, src/align.rs:216-222);
 *   * the gate score >= min_diag_score (:1638-1640), the region of the used
 *     segments (region, :1269-1278) when asked for, else [0, u32::MAX];
 *   * candidates ranked by score descending, then target ascending, cut to
 *     max_candidates (:1074-1083).
 *
 * With simd = 1 the job scores come from the AVX2 batched Kadane of
 * kadane_avx2.c (the reference's default path), and segment positions are
 * computed only for the chain pairs that could change the result, as the
 * reference does; with simd = 0 every job is scored by kadane_segment.  Both
 * give the same candidates.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

typedef struct {
  uint32_t t;
  int32_t d;
  uint32_t qpos;
  uint32_t idx;
} gate_hit;

static int cmp_hit(const void* a, const void* b) {
  const gate_hit* x = (const gate_hit*)a;
  const gate_hit* y = (const gate_hit*)b;
  if (x->t != y->t) return x->t < y->t ? -1 : 1;
  if (x->d != y->d) return x->d < y->d ? -1 : 1;
  return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

typedef struct {
  int64_t diag;
  uint32_t count, qmin, qmax;
} diag_run;

/* src/prefilter.rs:1194-1225: runs in ascending diagonal order; a run is
 * inserted before the first entry with a smaller count; at most kmax kept. */
static uint32_t top_diagonals(const gate_hit* g, uint32_t n, uint32_t kmax, diag_run* top) {
  uint32_t nt = 0;
  uint32_t a = 0;
  while (a < n) {
    diag_run r = {g[a].d, 0, g[a].qpos, g[a].qpos};
    uint32_t b = a;
    while (b < n && g[b].d == g[a].d) {
      if (g[b].qpos < r.qmin) r.qmin = g[b].qpos;
      if (g[b].qpos > r.qmax) r.qmax = g[b].qpos;
      ++b;
    }
    r.count = b - a;
    a = b;
    uint32_t pos = 0;
    while (pos < nt && !(r.count > top[pos].count)) ++pos;
    if (pos < kmax) {
      uint32_t last = nt < kmax ? nt : kmax - 1;
      for (uint32_t i = last; i > pos; --i) top[i] = top[i - 1];
      top[pos] = r;
      if (nt < kmax) ++nt;
    }
  }
  return nt;
}

static int32_t gap_cost(int32_t open, int32_t ext, uint64_t len) {
  return len == 0 ? 0 : (int32_t)((uint32_t)open + (uint32_t)((int32_t)len - 1) * (uint32_t)ext);
}

static int cmp_cand(const void* a, const void* b) {
  const or_candidate* x = (const or_candidate*)a;
  const or_candidate* y = (const or_candidate*)b;
  if (x->diag_score != y->diag_score) return x->diag_score > y->diag_score ? -1 : 1;
  return x->target < y->target ? -1 : (x->target > y->target);
}

uint64_t or_prefilter_query(const int32_t* rows, uint32_t m, uint32_t query, const uint8_t* tgt_arena,
                            const uint64_t* tgt_off, const uint32_t* ht, const int32_t* hd, const uint32_t* hqpos,
                            uint64_t n_hits, const or_prefilter_params* p, int simd, or_candidate* out,
                            or_prefilter_stats* st) {
  memset(st, 0, sizeof *st);
  if (n_hits == 0) return 0;
  gate_hit* h = (gate_hit*)malloc(n_hits * sizeof(gate_hit));
  for (uint64_t k = 0; k < n_hits; ++k) h[k] = (gate_hit){ht[k], hd[k], hqpos[k], (uint32_t)k};
  qsort(h, n_hits, sizeof(gate_hit), cmp_hit);
  const uint32_t kmax = p->max_diagonals ? p->max_diagonals : 1;
  diag_run* top = (diag_run*)malloc(kmax * sizeof(diag_run));
  /* jobs of every kept target, then scores in one batch (the reference flushes
   * every EV_CHUNK jobs, which changes nothing in the results) */
  uint64_t cap = n_hits;
  uint32_t* jt = (uint32_t*)malloc(cap * sizeof(uint32_t));
  int64_t* jd = (int64_t*)malloc(cap * sizeof(int64_t));
  uint32_t* jlo = (uint32_t*)malloc(cap * sizeof(uint32_t));
  uint32_t* jhi = (uint32_t*)malloc(cap * sizeof(uint32_t));
  uint32_t* tgt = (uint32_t*)malloc(cap * sizeof(uint32_t));
  uint32_t* tgt_hits = (uint32_t*)malloc(cap * sizeof(uint32_t));
  uint64_t* tgt_j0 = (uint64_t*)malloc((cap + 1) * sizeof(uint64_t));
  uint64_t nj = 0, ntg = 0;
  uint64_t i = 0;
  while (i < n_hits) {
    uint64_t j = i + 1;
    while (j < n_hits && h[j].t == h[i].t) ++j;
    st->targets_hit++;
    const uint32_t tid = h[i].t;
    const uint32_t gn = (uint32_t)(j - i);
    const gate_hit* g = h + i;
    i = j;
    if (gn < p->min_hits) continue;
    uint32_t nt = top_diagonals(g, gn, kmax, top);
    if (top[0].count < p->diag_hits) continue;
    st->targets_evaluated++;
    const uint64_t tn = tgt_off[tid + 1] - tgt_off[tid];
    tgt[ntg] = tid;
    tgt_hits[ntg] = gn;
    tgt_j0[ntg] = nj;
    for (uint32_t k = 0; k < nt && k < 16; ++k) {
      uint64_t lo, hi;
      or_diag_range(m, tn, top[k].diag, &lo, &hi);
      if (p->diag_window > 0) {
        const uint64_t a = top[k].qmin > p->diag_window ? top[k].qmin - p->diag_window : 0;
        const uint64_t b = (uint64_t)top[k].qmax + p->span + p->diag_window;
        if (a > lo) lo = a;
        if (b < hi) hi = b;
      }
      if (hi < lo) hi = lo;
      jt[nj] = tid;
      jd[nj] = top[k].diag;
      jlo[nj] = (uint32_t)lo;
      jhi[nj] = (uint32_t)hi;
      ++nj;
    }
    ++ntg;
  }
  tgt_j0[ntg] = nj;
  st->diagonals_scored = nj;
  int32_t* sc = (int32_t*)malloc((nj + 1) * sizeof(int32_t));
  uint64_t* qs = (uint64_t*)malloc((nj + 1) * sizeof(uint64_t));
  uint64_t* qe = (uint64_t*)malloc((nj + 1) * sizeof(uint64_t));
  uint8_t* have = (uint8_t*)calloc(nj + 1, 1);
  if (simd && nj) {
    const uint8_t** tp = (const uint8_t**)malloc(nj * sizeof(uint8_t*));
    for (uint64_t k = 0; k < nj; ++k) tp[k] = tgt_arena + tgt_off[jt[k]];
    or_kadane_jobs_avx2(rows, m, tp, jd, jlo, jhi, (uint32_t)nj, sc);
    free(tp);
  } else {
    for (uint64_t k = 0; k < nj; ++k) {
      sc[k] = or_kadane_segment(rows, tgt_arena + tgt_off[jt[k]], jd[k], jlo[k], jhi[k], &qs[k], &qe[k]);
      have[k] = 1;
    }
  }
#define POS_OF(k)                                                                                           \
  do {                                                                                                      \
    if (!have[k]) {                                                                                         \
      or_kadane_segment(rows, tgt_arena + tgt_off[jt[k]], jd[k], jlo[k], jhi[k], &qs[k], &qe[k]);           \
      have[k] = 1;                                                                                          \
    }                                                                                                       \
  } while (0)
  uint64_t nc = 0;
  for (uint64_t g = 0; g < ntg; ++g) {
    const uint64_t j0 = tgt_j0[g], ns = tgt_j0[g + 1] - j0;
    if (ns == 1 && sc[j0] < p->min_diag_score) continue;
    int32_t best = 0;
    uint64_t bi = 0;
    for (uint64_t k = 0; k < ns; ++k)
      if (sc[j0 + k] > best) {
        best = sc[j0 + k];
        bi = k;
      }
    int32_t chain = INT32_MIN;
    uint64_t cx = 0, cy = 0;
    if (ns > 1)
      for (uint64_t x = 0; x < ns; ++x)
        for (uint64_t y = 0; y < ns; ++y) {
          if (x == y) continue;
          const int32_t sx = sc[j0 + x], sy = sc[j0 + y];
          const int64_t dx = jd[j0 + x], dy = jd[j0 + y];
          if (sx <= 0 || sy <= 0 || dx == dy) continue;
          const uint64_t len = (uint64_t)(dy > dx ? dy - dx : dx - dy);
          const int32_t c =
              (int32_t)((uint32_t)sx + (uint32_t)sy - (uint32_t)gap_cost(p->gap_open, p->gap_ext, len));
          if (c <= best || c <= chain) continue;
          POS_OF(j0 + x);
          POS_OF(j0 + y);
          const int64_t qex = (int64_t)qe[j0 + x], qsy = (int64_t)qs[j0 + y];
          if (qex < qsy && qex + dx < qsy + dy) {
            chain = c;
            cx = x;
            cy = y;
          }
        }
    int32_t score;
    uint64_t used[2];
    if (chain > best) {
      st->chains_used++;
      score = chain;
      used[0] = cx;
      used[1] = cy;
    } else {
      score = best;
      used[0] = used[1] = bi;
    }
    if (score < p->min_diag_score) continue;
    uint32_t rlo = 0, rhi = UINT32_MAX;
    if (p->regions) {
      rlo = UINT32_MAX;
      rhi = 0;
      for (int u = 0; u < 2; ++u) {
        const uint64_t k = j0 + used[u];
        POS_OF(k);
        const int64_t a = (int64_t)qs[k] + jd[k], b = (int64_t)qe[k] + jd[k];
        const uint32_t la = (uint32_t)(a > 0 ? a : 0), lb = (uint32_t)(b > 0 ? b : 0);
        if (la < rlo) rlo = la;
        if (lb > rhi) rhi = lb;
      }
    }
    out[nc++] = (or_candidate){query, tgt[g], tgt_hits[g], score, jd[j0 + bi], rlo, rhi};
  }
#undef POS_OF
  qsort(out, nc, sizeof(or_candidate), cmp_cand);
  if (p->max_candidates > 0 && nc > p->max_candidates) {
    st->candidates_capped = nc - p->max_candidates;
    nc = p->max_candidates;
  }
  st->candidates = nc;
  free(h);
  free(top);
  free(jt);
  free(jd);
  free(jlo);
  free(jhi);
  free(tgt);
  free(tgt_hits);
  free(tgt_j0);
  free(sc);
  free(qs);
  free(qe);
  free(have);
  return nc;
}

void or_prefilter_queries(const int32_t* rows_arena, const uint64_t* row_off, const uint32_t* qlen,
                          const uint32_t* qids, uint32_t n_queries, const uint8_t* tgt_arena, const uint64_t* tgt_off,
                          const uint64_t* hstart, const uint32_t* ht, const int32_t* hd, const uint32_t* hqpos,
                          const or_prefilter_params* p, int simd, or_candidate* out, uint64_t* n_out,
                          or_prefilter_stats* stats, int nthreads) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
  for (int64_t q = 0; q < (int64_t)n_queries; ++q) {
    const uint32_t id = qids[q];
    const uint64_t a = hstart[q], b = hstart[q + 1];
    n_out[q] = or_prefilter_query(rows_arena + row_off[id] * OR_NPROF, qlen[id], id, tgt_arena, tgt_off, ht + a,
                                  hd + a, hqpos + a, b - a, p, simd, out + a, stats + q);
  }
}
