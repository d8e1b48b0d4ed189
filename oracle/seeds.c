/*
 * Seed hits — TEST/BENCH INFRASTRUCTURE ONLY.  A plain-C restatement of the
 * reference's seed stage of prefilter_query (src/prefilter.rs:816-995):
 *
 *   * every window start of the query, start in [0, m - span]; a window whose
 *     care positions hold a residue code >= 20 is skipped (sequence queries);
 *   * its similar k-mers: the first `cap` k-mers with score >= threshold in the
 *     canonical order (score descending, then the rank vector — each position's
 *     residues ranked by score descending, residue ascending — ascending),
 *     restated from the reference's best-first generator top_kmers_heap
 *     (:624-690), which its tests use as the oracle of top_kmers (:1754-1837);
 *   * the query's own k-mer added when exact_seeds is set and it is not among
 *     them (:974-983);
 *   * each k-mer's postings in the seed index — every target window whose care
 *     residues are all < 20 (window_ok, src/index.rs:1059-1074), code = care
 *     residues in base 20 — skipped when longer than max_seed_occ (push_seed,
 *     :853-869); a posting (target, tpos) is the hit (target, tpos - qpos, qpos).
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define AA 20
#define MAXK 12

typedef struct {
  int32_t score;
  uint64_t code;
  uint8_t ranks[MAXK];
  uint8_t last;
} kitem;

typedef struct {
  int32_t sc[AA];
  uint8_t res[AA];
} srow;

/* sorted_row (src/prefilter.rs:433-441) */
static void sort_row(const int32_t* row, srow* out) {
  for (int r = 0; r < AA; ++r) {
    out->sc[r] = row[r];
    out->res[r] = (uint8_t)r;
  }
  for (int i = 1; i < AA; ++i) /* stable insertion sort: score descending, residue ascending */
    for (int j = i; j > 0 && out->sc[j] > out->sc[j - 1]; --j) {
      int32_t ts = out->sc[j];
      out->sc[j] = out->sc[j - 1];
      out->sc[j - 1] = ts;
      uint8_t tr = out->res[j];
      out->res[j] = out->res[j - 1];
      out->res[j - 1] = tr;
    }
}

/* heap order: higher score first; equal scores: lexicographically smaller rank vector first */
static int kbefore(const kitem* a, const kitem* b, int w) {
  if (a->score != b->score) return a->score > b->score;
  return memcmp(a->ranks, b->ranks, (size_t)w) < 0;
}

static void kpush(kitem* h, uint32_t* n, kitem it, int w) {
  uint32_t i = (*n)++;
  h[i] = it;
  while (i > 0) {
    uint32_t p = (i - 1) / 2;
    if (!kbefore(&h[i], &h[p], w)) break;
    kitem t = h[i];
    h[i] = h[p];
    h[p] = t;
    i = p;
  }
}

static kitem kpop(kitem* h, uint32_t* n, int w) {
  kitem top = h[0];
  h[0] = h[--(*n)];
  uint32_t i = 0;
  for (;;) {
    uint32_t l = 2 * i + 1, r = l + 1, b = i;
    if (l < *n && kbefore(&h[l], &h[b], w)) b = l;
    if (r < *n && kbefore(&h[r], &h[b], w)) b = r;
    if (b == i) break;
    kitem t = h[i];
    h[i] = h[b];
    h[b] = t;
    i = b;
  }
  return top;
}

static int top_kmers_sorted(const srow* rows, int w, int32_t thr, uint32_t cap, uint64_t* codes, int32_t* scores,
                            uint32_t* n_out) {
  *n_out = 0;
  if (w == 0 || cap == 0) return 0;
  int32_t s0 = 0;
  for (int i = 0; i < w; ++i) s0 += rows[i].sc[0];
  if (s0 < thr) return 0;
  kitem* heap = (kitem*)malloc(((size_t)cap * w + 2) * sizeof(kitem));
  uint32_t hn = 0;
  kitem it;
  memset(&it, 0, sizeof it);
  it.score = s0;
  for (int i = 0; i < w; ++i) it.code = it.code * AA + rows[i].res[0];
  kpush(heap, &hn, it, w);
  int capped = 0;
  while (hn > 0) {
    kitem x = kpop(heap, &hn, w);
    if (*n_out >= cap) {
      capped = 1;
      break;
    }
    codes[*n_out] = x.code;
    scores[*n_out] = x.score;
    (*n_out)++;
    for (int j = x.last; j < w; ++j) {
      const int r = x.ranks[j];
      if (r + 1 >= AA) continue;
      const int32_t ns = x.score - rows[j].sc[r] + rows[j].sc[r + 1];
      if (ns < thr) continue;
      kitem y = x;
      y.ranks[j]++;
      y.last = (uint8_t)j;
      y.score = ns;
      y.code = 0;
      for (int i = 0; i < w; ++i) y.code = y.code * AA + rows[i].res[y.ranks[i]];
      kpush(heap, &hn, y, w);
    }
  }
  free(heap);
  return capped;
}

/* cap_boundary (src/prefilter.rs:571-609): the largest score t with at least cap
 * k-mers >= t among those >= thr, and how many score above t. */
static void cap_boundary(const srow* rows, int w, const int32_t* smax, int32_t thr, uint32_t cap, int32_t* t_out,
                         uint64_t* above_out) {
  /* histograms of partial sums pruned at the threshold (u64 counts) */
  int32_t lo = 0, hi = 0;
  size_t n = 1;
  uint64_t* dist = (uint64_t*)calloc(1, sizeof(uint64_t));
  dist[0] = 1;
  for (int i = 0; i < w; ++i) {
    const int32_t nhi = hi + rows[i].sc[0];
    int32_t nlo = lo + rows[i].sc[AA - 1];
    const int32_t need = thr - smax[i + 1];
    if (need > nlo) nlo = need;
    const size_t nn = (size_t)(nhi - nlo + 1);
    uint64_t* tmp = (uint64_t*)calloc(nn, sizeof(uint64_t));
    for (size_t off = 0; off < n; ++off) {
      const uint64_t cnt = dist[off];
      if (!cnt) continue;
      const int32_t sv = lo + (int32_t)off;
      for (int a = 0; a < AA; ++a) {
        const int32_t t = sv + rows[i].sc[a];
        if (t < nlo) break;
        tmp[t - nlo] += cnt;
      }
    }
    free(dist);
    dist = tmp;
    n = nn;
    lo = nlo;
    hi = nhi;
  }
  uint64_t above = 0;
  int32_t t = hi;
  for (;; --t) {
    const uint64_t c = dist[t - lo];
    if (above + c >= cap) break;
    above += c;
  }
  free(dist);
  *t_out = t;
  *above_out = above;
}

/* top_kmers (src/prefilter.rs:470-568), the reference's default generator: a
 * depth-first walk in rank-lexicographic order with suffix-maximum pruning;
 * past the cap, the boundary score t* from cap_boundary, the list cut to the
 * k-mers above t* plus the first ties, and only those accepted from then on.
 * The returned set equals top_kmers_heap's; its order is the walk's. */
static int top_kmers_dfs(const srow* rows, int w, int32_t thr, uint32_t cap, uint64_t* codes, int32_t* scores,
                         uint32_t* n_out) {
  *n_out = 0;
  if (w == 0 || cap == 0) return 0;
  int32_t smax[MAXK + 1];
  smax[w] = 0;
  for (int i = w - 1; i >= 0; --i) smax[i] = smax[i + 1] + rows[i].sc[0];
  if (smax[0] < thr) return 0;
  int32_t th = thr, tstar = INT32_MIN;
  int capped = 0;
  uint64_t ties_left = 0;
  const int last = w - 1;
  uint8_t rank[MAXK] = {0};
  int32_t part[MAXK + 1] = {0};
  uint64_t code[MAXK + 1] = {0};
  uint32_t n = 0;
  int d = 0;
  for (;;) {
    if (d == last) {
      const int32_t bs = part[last];
      const uint64_t bc = code[last] * AA;
      for (int a = 0; a < AA; ++a) {
        const int32_t ns = bs + rows[last].sc[a];
        if (ns < th) break;
        /* the buffer holds at most cap + 1 entries: cut as soon as it passes cap */
        codes[n] = bc + rows[last].res[a];
        scores[n] = ns;
        ++n;
        if (capped) {
          if (ns == tstar && --ties_left == 0) th = tstar + 1;
        } else if (n > cap) {
          capped = 1;
          uint64_t above;
          cap_boundary(rows, w, smax, th, cap, &tstar, &above);
          const uint64_t need = cap - above;
          uint64_t kept = 0;
          uint32_t k2 = 0;
          for (uint32_t k = 0; k < n; ++k) {
            if (scores[k] > tstar || (scores[k] == tstar && kept < need)) {
              if (scores[k] == tstar) ++kept;
              codes[k2] = codes[k];
              scores[k2] = scores[k];
              ++k2;
            }
          }
          n = k2;
          ties_left = need - kept;
          th = ties_left == 0 ? tstar + 1 : tstar;
        }
      }
      if (last == 0) break;
      d = last - 1;
      ++rank[d];
      continue;
    }
    const int r = rank[d];
    if (r < AA) {
      const int32_t ns = part[d] + rows[d].sc[r];
      if (ns + smax[d + 1] >= th) {
        part[d + 1] = ns;
        code[d + 1] = code[d] * AA + rows[d].res[r];
        ++d;
        rank[d] = 0;
        continue;
      }
    }
    if (d == 0) break;
    --d;
    ++rank[d];
  }
  *n_out = n;
  return capped;
}

int or_top_kmers_dfs(const int32_t* rows, int w, int32_t thr, uint32_t cap, uint64_t* codes, int32_t* scores,
                     uint32_t* n_out) {
  srow sr[MAXK];
  for (int i = 0; i < w && i < MAXK; ++i) sort_row(rows + (size_t)i * OR_NPROF, &sr[i]);
  return top_kmers_dfs(sr, w, thr, cap, codes, scores, n_out);
}

int or_top_kmers(const int32_t* rows, int w, int32_t thr, uint32_t cap, uint64_t* codes, int32_t* scores,
                 uint32_t* n_out) {
  srow sr[MAXK];
  for (int i = 0; i < w && i < MAXK; ++i) sort_row(rows + (size_t)i * OR_NPROF, &sr[i]);
  return top_kmers_sorted(sr, w, thr, cap, codes, scores, n_out);
}

static int cmp_post(const void* a, const void* b) {
  const or_posting* x = (const or_posting*)a;
  const or_posting* y = (const or_posting*)b;
  if (x->code != y->code) return x->code < y->code ? -1 : 1;
  if (x->tid != y->tid) return x->tid < y->tid ? -1 : 1;
  return x->tpos < y->tpos ? -1 : (x->tpos > y->tpos);
}

uint64_t or_index_count(const uint8_t* tgt_arena, const uint64_t* tgt_off, uint32_t n_targets, const uint32_t* offs,
                        uint32_t w, uint32_t span) {
  uint64_t n = 0;
  for (uint32_t t = 0; t < n_targets; ++t) {
    const uint8_t* s = tgt_arena + tgt_off[t];
    const uint64_t len = tgt_off[t + 1] - tgt_off[t];
    if (len < span) continue;
    for (uint64_t st = 0; st + span <= len; ++st) {
      int ok = 1;
      for (uint32_t i = 0; i < w; ++i)
        if (s[st + offs[i]] >= AA) ok = 0;
      n += (uint64_t)ok;
    }
  }
  return n;
}

void or_index_build(const uint8_t* tgt_arena, const uint64_t* tgt_off, uint32_t n_targets, const uint32_t* offs,
                    uint32_t w, uint32_t span, or_posting* out) {
  uint64_t n = 0;
  for (uint32_t t = 0; t < n_targets; ++t) {
    const uint8_t* s = tgt_arena + tgt_off[t];
    const uint64_t len = tgt_off[t + 1] - tgt_off[t];
    if (len < span) continue;
    for (uint64_t st = 0; st + span <= len; ++st) {
      uint64_t code = 0;
      int ok = 1;
      for (uint32_t i = 0; i < w; ++i) {
        const uint8_t r = s[st + offs[i]];
        if (r >= AA) ok = 0;
        code = code * AA + r;
      }
      if (ok) out[n++] = (or_posting){code, t, (uint32_t)st};
    }
  }
  qsort(out, n, sizeof(or_posting), cmp_post);
}

static void post_range(const or_posting* idx, uint64_t n, uint64_t code, uint64_t* a, uint64_t* b) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    uint64_t mid = (lo + hi) / 2;
    if (idx[mid].code < code) lo = mid + 1; else hi = mid;
  }
  *a = lo;
  hi = n;
  while (lo < hi) {
    uint64_t mid = (lo + hi) / 2;
    if (idx[mid].code <= code) lo = mid + 1; else hi = mid;
  }
  *b = lo;
}

uint64_t or_seed_hits(const int32_t* rows, const uint8_t* residues, uint32_t m, const uint32_t* offs, uint32_t w,
                      uint32_t span, const or_seed_params* p, const or_posting* idx, uint64_t n_post, uint32_t query,
                      uint32_t* ht, int32_t* hd, uint32_t* hqpos, uint64_t cap_hits, or_seed_stats* st) {
  memset(st, 0, sizeof *st);
  if (m < span || n_post == 0 || w == 0 || w > MAXK) return 0;
  (void)query;
  srow* sr = (srow*)malloc((size_t)m * sizeof(srow));
  for (uint32_t i = 0; i < m; ++i) sort_row(rows + (size_t)i * OR_NPROF, &sr[i]);
  const uint32_t kcap = p->max_kmers_per_pos;
  uint64_t* codes = (uint64_t*)malloc(((size_t)kcap + 1) * sizeof(uint64_t));
  int32_t* scores = (int32_t*)malloc(((size_t)kcap + 1) * sizeof(int32_t));
  uint64_t nh = 0;
  for (uint32_t start = 0; start + span <= m; ++start) {
    st->windows++;
    int skip = 0;
    uint64_t exact = 0;
    srow wr[MAXK];
    for (uint32_t i = 0; i < w; ++i) {
      const uint32_t c = start + offs[i];
      if (residues) {
        if (residues[c] >= AA) {
          skip = 1;
          break;
        }
        exact = exact * AA + residues[c];
      }
      wr[i] = sr[c];
    }
    if (skip) {
      st->windows_skipped++;
      continue;
    }
    uint32_t nk = 0;
    const int at_cap = top_kmers_sorted(wr, (int)w, p->kmer_score, kcap, codes, scores, &nk);
    st->windows_at_cap += (uint64_t)at_cap;
    int have_exact = 0;
    for (uint32_t k = 0; k < nk; ++k) have_exact |= codes[k] == exact;
    const int add_exact = residues && p->exact_seeds && !have_exact;
    if (add_exact) {
      codes[nk++] = exact;
      st->exact_seeds_added++;
    }
    st->kmers_generated += nk;
    for (uint32_t k = 0; k < nk; ++k) {
      uint64_t a, b;
      post_range(idx, n_post, codes[k], &a, &b);
      if (b <= a) continue;
      if (p->max_seed_occ > 0 && b - a > p->max_seed_occ) {
        st->seeds_over_occ_cap++;
        st->postings_skipped_occ += b - a;
        continue;
      }
      st->seeds++;
      st->postings_visited += b - a;
      for (uint64_t e = a; e < b; ++e) {
        if (nh < cap_hits) {
          ht[nh] = idx[e].tid;
          hd[nh] = (int32_t)((int64_t)idx[e].tpos - (int64_t)start);
          hqpos[nh] = start;
        }
        ++nh;
      }
    }
  }
  free(sr);
  free(codes);
  free(scores);
  return nh;
}

/* ---- direct-table index and batched queries (the CPU baseline of the search) ----
 * The same index as or_index_build as a direct table: off[code] .. off[code+1]
 * indexes post (target, position) pairs, built by a counting sort over all
 * windows (20^w + 1 offsets, w <= 7). */
uint64_t or_index_direct_build(const uint8_t* tgt_arena, const uint64_t* tgt_off, uint32_t n_targets,
                               const uint32_t* offs, uint32_t w, uint32_t span, uint64_t* off, uint32_t* post_t,
                               uint32_t* post_p, int count_only) {
  uint64_t n_codes = 1;
  for (uint32_t i = 0; i < w; ++i) n_codes *= AA;
  if (count_only) memset(off, 0, (n_codes + 1) * sizeof(uint64_t));
  for (uint32_t t = 0; t < n_targets; ++t) {
    const uint8_t* s = tgt_arena + tgt_off[t];
    const uint64_t len = tgt_off[t + 1] - tgt_off[t];
    if (len < span) continue;
    for (uint64_t st = 0; st + span <= len; ++st) {
      uint64_t code = 0;
      int ok = 1;
      for (uint32_t i = 0; i < w; ++i) {
        const uint8_t r = s[st + offs[i]];
        if (r >= AA) ok = 0;
        code = code * AA + r;
      }
      if (!ok) continue;
      if (count_only) {
        off[code + 1]++;
      } else {
        const uint64_t k = off[code]++;
        post_t[k] = t;
        post_p[k] = (uint32_t)st;
      }
    }
  }
  if (count_only)
    for (uint64_t c = 0; c < n_codes; ++c) off[c + 1] += off[c];
  return off[n_codes];
}

/* Queries in parallel over the direct index (off already shifted back: off[c] is
 * the start of code c): seed hits as or_seed_hits, then the evidence stage of
 * or_prefilter_query.  n_cand[q] receives each query's candidate count; at most
 * cap_per_query candidates of query q are written at out + q * cap_per_query. */
void or_prefilter_search(const int32_t* rows_arena, const uint64_t* row_off, const uint32_t* qlen,
                         const uint8_t* res_arena, uint32_t n_queries, const uint8_t* tgt_arena,
                         const uint64_t* tgt_off, const uint32_t* offs, uint32_t w, uint32_t span,
                         const uint64_t* off, const uint32_t* post_t, const uint32_t* post_p,
                         const or_seed_params* sp, const or_prefilter_params* gp, or_candidate* out,
                         uint64_t cap_per_query, uint64_t* n_cand, uint64_t* n_hits, int nthreads) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
  for (int64_t q = 0; q < (int64_t)n_queries; ++q) {
    const int32_t* rows = rows_arena + row_off[q] * OR_NPROF;
    const uint32_t m = qlen[q];
    const uint8_t* res = res_arena ? res_arena + row_off[q] : NULL;
    n_cand[q] = 0;
    n_hits[q] = 0;
    if (m < span) continue;
    srow* sr = (srow*)malloc((size_t)m * sizeof(srow));
    for (uint32_t i = 0; i < m; ++i) sort_row(rows + (size_t)i * OR_NPROF, &sr[i]);
    uint64_t* codes = (uint64_t*)malloc(((size_t)sp->max_kmers_per_pos + 2) * sizeof(uint64_t));
    int32_t* scores = (int32_t*)malloc(((size_t)sp->max_kmers_per_pos + 2) * sizeof(int32_t));
    uint64_t cap_h = 1 << 16, nh = 0;
    uint32_t* ht = (uint32_t*)malloc(cap_h * 4);
    int32_t* hd = (int32_t*)malloc(cap_h * 4);
    uint32_t* hq = (uint32_t*)malloc(cap_h * 4);
    for (uint32_t start = 0; start + span <= m; ++start) {
      srow wr[MAXK];
      uint64_t exact = 0;
      int skip = 0;
      for (uint32_t i = 0; i < w; ++i) {
        const uint32_t c = start + offs[i];
        if (res) {
          if (res[c] >= AA) {
            skip = 1;
            break;
          }
          exact = exact * AA + res[c];
        }
        wr[i] = sr[c];
      }
      if (skip) continue;
      uint32_t nk = 0;
      top_kmers_dfs(wr, (int)w, sp->kmer_score, sp->max_kmers_per_pos, codes, scores, &nk);
      int have = 0;
      for (uint32_t k = 0; k < nk; ++k) have |= codes[k] == exact;
      if (res && sp->exact_seeds && !have) codes[nk++] = exact;
      for (uint32_t k = 0; k < nk; ++k) {
        const uint64_t a = off[codes[k]], b = off[codes[k] + 1];
        if (b <= a || (sp->max_seed_occ > 0 && b - a > sp->max_seed_occ)) continue;
        if (nh + (b - a) > cap_h) {
          while (nh + (b - a) > cap_h) cap_h *= 2;
          ht = (uint32_t*)realloc(ht, cap_h * 4);
          hd = (int32_t*)realloc(hd, cap_h * 4);
          hq = (uint32_t*)realloc(hq, cap_h * 4);
        }
        for (uint64_t e = a; e < b; ++e) {
          ht[nh] = post_t[e];
          hd[nh] = (int32_t)post_p[e] - (int32_t)start;
          hq[nh] = start;
          ++nh;
        }
      }
    }
    n_hits[q] = nh;
    if (nh) {
      or_candidate* tmp = (or_candidate*)malloc(nh * sizeof(or_candidate));
      or_prefilter_stats st;
      const uint64_t nc =
          or_prefilter_query(rows, m, (uint32_t)q, tgt_arena, tgt_off, ht, hd, hq, nh, gp, 1, tmp, &st);
      n_cand[q] = nc;
      memcpy(out + (size_t)q * cap_per_query, tmp, (nc < cap_per_query ? nc : cap_per_query) * sizeof(or_candidate));
      free(tmp);
    }
    free(sr);
    free(codes);
    free(scores);
    free(ht);
    free(hd);
    free(hq);
  }
}
