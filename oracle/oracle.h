/*
 * CPU oracle for the Sabertooth alignment hot path — TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference's scalar (exact) kernels, used
 * as the checker for the CUDA path and, in bench.py's CPU-baseline leg only, as
 * the timed CPU baseline.  Nothing in the product (the sabertooth_b200 package
 * or libsabertooth_b200.so) may link, import or call it.
 *
 * Reference (raw-lab/sabertooth v0.4.0, Rust), followed line by line:
 *   diag_range          src/ungapped.rs:38-46
 *   kadane_score        src/ungapped.rs:53-62
 *   kadane_segment      src/ungapped.rs:69-88
 *   gotoh_score_end     src/simd.rs:347-390   (scalar_gotoh_score_end, column-major-first end)
 *   gotoh_score         src/simd.rs:252-255, 342-345 (m == 0 or empty target -> 0)
 *   reference_score     src/simd.rs:1124-1142 and src/align.rs:1150-1166 (three full matrices)
 *   band_score          src/align.rs:408-493  (local_full_tb with band = Some((center, radius)))
 *
 * Score rows are the reference's ScoreTable rows: int32 [m][21], residue codes
 * 0..20 (A..Y, X); target codes >= 21 score 0 (src/align.rs:180-186,
 * src/simd.rs:367-368).  Parity pins: see tests/test_oracle.py.
 */
#ifndef SABERTOOTH_ORACLE_H
#define SABERTOOTH_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define OR_NPROF 21

void or_diag_range(uint64_t m, uint64_t n, int64_t d, uint64_t* lo, uint64_t* hi);
int32_t or_kadane_score(const int32_t* rows, const uint8_t* t, int64_t d, uint64_t lo, uint64_t hi);
int32_t or_kadane_segment(const int32_t* rows, const uint8_t* t, int64_t d, uint64_t lo, uint64_t hi,
                          uint64_t* q_start, uint64_t* q_end);

/* returns 1 and fills (score, query_end, target_end) when best > 0, else 0 */
int or_gotoh_score_end(const int32_t* rows, uint32_t m, const uint8_t* t, uint32_t n, int32_t open,
                       int32_t ext, int32_t* score, uint32_t* qi, uint32_t* tj);
int32_t or_gotoh_score(const int32_t* rows, uint32_t m, const uint8_t* t, uint32_t n, int32_t open,
                       int32_t ext);
int32_t or_reference_score(const int32_t* rows, uint32_t m, const uint8_t* t, uint32_t n, int32_t open,
                           int32_t ext);
int32_t or_band_score(const int32_t* rows, uint32_t m, const uint8_t* t, uint32_t n, int32_t open,
                      int32_t ext, int64_t center, int64_t radius);

/* Batched forms (OpenMP over pairs) for larger parity cases.
 * rows_arena: concatenated int32 [m_q][21] rows; row_off[q] = first row of query q; qlen[q] = m_q.
 * tgt_arena: concatenated target codes; tgt_off[t] .. tgt_off[t+1].
 * pair k = (pq[k], pt[k]); radius[k] < 0 -> full SW, else band (center[k], radius[k]). */
void or_sw_pairs(const int32_t* rows_arena, const uint64_t* row_off, const uint32_t* qlen,
                 const uint8_t* tgt_arena, const uint64_t* tgt_off, const uint32_t* pq, const uint32_t* pt,
                 const int64_t* center, const int64_t* radius, uint64_t n_pairs, int32_t open, int32_t ext,
                 int32_t* out, int nthreads);

/* hit k = (hq[k], ht[k], hd[k]); score over the whole diagonal (diag_range). */
void or_ungapped_hits(const int32_t* rows_arena, const uint64_t* row_off, const uint32_t* qlen,
                      const uint8_t* tgt_arena, const uint64_t* tgt_off, const uint32_t* hq, const uint32_t* ht,
                      const int32_t* hd, uint64_t n_hits, int32_t* out, int nthreads);
/* The reference's AVX2 batched Kadane over seed-hit diagonals (kadane_avx2.c): the CPU baseline of (U). */
void or_ungapped_hits_avx2(const int32_t* rows_arena, const uint64_t* row_off, const uint32_t* qlen,
                           const uint8_t* tgt_arena, const uint64_t* tgt_off, const uint32_t* hq, const uint32_t* ht,
                           const int32_t* hd, uint64_t n_hits, int32_t* out, int nthreads);

/* CPU baseline (striped.c): the reference's default AVX2 path (u8 striped -> i16 striped ->
 * scalar) over pairs grouped by query; query q's targets are tlist[qstart[q] .. qstart[q+1]).
 * used[k] (may be NULL): 1 = u8 pass decided, 2 = i16, 3 = scalar, 0 = empty input. */
void or_striped_queries(const int32_t* rows_arena, const uint64_t* row_off, const uint32_t* qlen, uint32_t n_queries,
                        const uint8_t* tgt_arena, const uint64_t* tgt_off, const uint64_t* qstart,
                        const uint32_t* tlist, int32_t open, int32_t ext, int32_t* out, uint8_t* used,
                        int nthreads);

/* ---- prefilter evidence, chain and gate (gate.c) ----------------------------
 * One query's seed hits (target, diagonal = target_pos - query_pos, query
 * position) -> ranked candidates: the segment-evidence stage of prefilter_query
 * (src/prefilter.rs:1412-1660, ranking :1074-1083).  out needs room for one
 * candidate per distinct target (n_hits suffices). */
typedef struct {
  uint32_t query;
  uint32_t target;
  uint32_t hits;
  int32_t diag_score;
  int64_t best_diag;
  uint32_t t_lo;
  uint32_t t_hi;
} or_candidate;

typedef struct {
  uint32_t min_hits;
  uint32_t diag_hits;
  uint32_t max_diagonals;
  uint32_t diag_window;
  uint32_t span;
  int32_t min_diag_score;
  int32_t gap_open;
  int32_t gap_ext;
  uint32_t max_candidates;
  uint32_t regions;
} or_prefilter_params;

typedef struct {
  uint64_t targets_hit;
  uint64_t targets_evaluated;
  uint64_t diagonals_scored;
  uint64_t chains_used;
  uint64_t candidates;
  uint64_t candidates_capped;
} or_prefilter_stats;

uint64_t or_prefilter_query(const int32_t* rows, uint32_t m, uint32_t query, const uint8_t* tgt_arena,
                            const uint64_t* tgt_off, const uint32_t* ht, const int32_t* hd, const uint32_t* hqpos,
                            uint64_t n_hits, const or_prefilter_params* p, int simd, or_candidate* out,
                            or_prefilter_stats* st);
/* Queries in parallel: query q (profile id qids[q]) owns hits hstart[q] .. hstart[q+1]
 * and writes n_out[q] candidates at out + hstart[q], stats[q] its counters. */
void or_prefilter_queries(const int32_t* rows_arena, const uint64_t* row_off, const uint32_t* qlen,
                          const uint32_t* qids, uint32_t n_queries, const uint8_t* tgt_arena, const uint64_t* tgt_off,
                          const uint64_t* hstart, const uint32_t* ht, const int32_t* hd, const uint32_t* hqpos,
                          const or_prefilter_params* p, int simd, or_candidate* out, uint64_t* n_out,
                          or_prefilter_stats* stats, int nthreads);
/* The AVX2 batched Kadane over one query's jobs with explicit windows (kadane_avx2.c). */
void or_kadane_jobs_avx2(const int32_t* rows, uint32_t m, const uint8_t* const* tp, const int64_t* d,
                         const uint32_t* lo, const uint32_t* hi, uint32_t n, int32_t* out);

/* ---- per-profile calibration (calib.c) ----------------------------------------
 * calibrate_profile (src/evalue.rs:714-748): background targets from per-sample
 * SplitMix64 streams, exact SW scores, ML Gumbel fit.  Returns 0 where the
 * reference returns None; scores[samples] are written whenever n_lengths and m
 * are non-zero. */
uint64_t or_stream_seed(uint64_t seed, uint64_t c, uint64_t i);
void or_background_cum(const double* p_back20, double* cum20);
uint32_t or_calibration_length(const uint32_t* lengths, uint32_t n_lengths, uint64_t seed, uint64_t i);
void or_calibration_target(const uint32_t* lengths, uint32_t n_lengths, uint64_t seed, uint64_t i, const double* cum20,
                           uint8_t* out, uint32_t* len);
double or_gumbel_mu_given_lambda(const double* xs, uint64_t n, double lambda);
int or_fit_gumbel_ml(const double* xs, uint64_t n, double* lambda, double* mu);
int or_calibrate_profile(const int32_t* rows, uint32_t m, const uint32_t* lengths, uint32_t n_lengths,
                         uint32_t samples, uint64_t seed, const double* p_back20, int32_t open, int32_t ext,
                         int32_t* scores, double* lambda, double* k, double* mu, int nthreads);

/* ---- seed hits (seeds.c) ---------------------------------------------------------
 * The seed stage of prefilter_query (src/prefilter.rs:816-995) over a CPU seed
 * index of the targets (window_ok, src/index.rs:1059-1074). */
typedef struct {
  uint64_t code;
  uint32_t tid;
  uint32_t tpos;
} or_posting;

typedef struct {
  int32_t kmer_score;
  uint32_t max_kmers_per_pos;
  uint32_t exact_seeds;
  uint32_t max_seed_occ; /* 0 = never skip */
} or_seed_params;

typedef struct {
  uint64_t windows;
  uint64_t windows_skipped;
  uint64_t kmers_generated;
  uint64_t windows_at_cap;
  uint64_t exact_seeds_added;
  uint64_t seeds;
  uint64_t postings_visited;
  uint64_t seeds_over_occ_cap;
  uint64_t postings_skipped_occ;
} or_seed_stats;

/* top_kmers_heap (src/prefilter.rs:624-690): rows = w x 21 score rows of the
 * window's care positions; codes/scores in canonical order (room for cap);
 * returns 1 when more than cap k-mers reach thr. */
int or_top_kmers(const int32_t* rows, int w, int32_t thr, uint32_t cap, uint64_t* codes, int32_t* scores,
                 uint32_t* n_out);
/* top_kmers (src/prefilter.rs:470-568), the reference's default depth-first generator with
 * cap_boundary: the same set as or_top_kmers in walk order; codes/scores need room for cap + 1. */
int or_top_kmers_dfs(const int32_t* rows, int w, int32_t thr, uint32_t cap, uint64_t* codes, int32_t* scores,
                     uint32_t* n_out);
uint64_t or_index_count(const uint8_t* tgt_arena, const uint64_t* tgt_off, uint32_t n_targets, const uint32_t* offs,
                        uint32_t w, uint32_t span);
/* out: room for or_index_count entries; sorted by (code, target, position) */
void or_index_build(const uint8_t* tgt_arena, const uint64_t* tgt_off, uint32_t n_targets, const uint32_t* offs,
                    uint32_t w, uint32_t span, or_posting* out);
/* one query's hits (target, diag, qpos), at most cap_hits written; returns the total.
 * residues may be NULL (profile queries: no skipped windows, no exact seeds). */
uint64_t or_seed_hits(const int32_t* rows, const uint8_t* residues, uint32_t m, const uint32_t* offs, uint32_t w,
                      uint32_t span, const or_seed_params* p, const or_posting* idx, uint64_t n_post, uint32_t query,
                      uint32_t* ht, int32_t* hd, uint32_t* hqpos, uint64_t cap_hits, or_seed_stats* st);
/* Direct-table index: count_only = 1 fills off (20^w + 1 entries, prefix sums:
 * off[c] = first posting of code c) and returns the postings; count_only = 0
 * fills post_t/post_p and advances off[c] to the end of each code (shift it back
 * by one entry, off[c] = old off[c-1], before lookups). */
uint64_t or_index_direct_build(const uint8_t* tgt_arena, const uint64_t* tgt_off, uint32_t n_targets,
                               const uint32_t* offs, uint32_t w, uint32_t span, uint64_t* off, uint32_t* post_t,
                               uint32_t* post_p, int count_only);
void or_prefilter_search(const int32_t* rows_arena, const uint64_t* row_off, const uint32_t* qlen,
                         const uint8_t* res_arena, uint32_t n_queries, const uint8_t* tgt_arena,
                         const uint64_t* tgt_off, const uint32_t* offs, uint32_t w, uint32_t span,
                         const uint64_t* off, const uint32_t* post_t, const uint32_t* post_p,
                         const or_seed_params* sp, const or_prefilter_params* gp, or_candidate* out,
                         uint64_t cap_per_query, uint64_t* n_cand, uint64_t* n_hits, int nthreads);

/* Sequence-query row preparation (rowprep.c): composition-bias correction
 * (src/compbias.rs:38-70) and the low-complexity mask (src/mask.rs:68-128). */
void or_comp_bias(const uint8_t* q, uint32_t n, const int32_t* score, const double* p_back, int penalize_only,
                  int32_t* out);
uint32_t or_low_complexity_mask(const uint8_t* seq, uint32_t n, uint32_t w, double locut, double hicut,
                                uint8_t* mask);

#ifdef __cplusplus
}
#endif
#endif
