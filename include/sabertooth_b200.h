/*
 * sabertooth_b200 — C ABI of the B200 (sm_100a) alignment hot path.
 *
 * Drop-in boundary for the reference crate raw-lab/sabertooth v0.4.0 (Rust).
 * Each entry point names the reference function it replaces (path:line in the
 * reference crate).  All entry points return an int status: ST_OK (0) on
 * success, a negative ST_E* code otherwise; st_last_error() returns a
 * thread-local message for the last failure on the calling thread.  The
 * reference functions are infallible, so a Rust shim turns a non-zero status
 * into a panic with that message; there is no CPU fallback.
 *
 * Conventions (as in the reference):
 *   - residue codes 0..20 (A C D E F G H I K L M N P Q R S T V W Y X,
 *     src/alphabet.rs:8-10); target codes >= 21 score 0 (src/align.rs:180-186);
 *   - score rows are int32 [m][21] ScoreTable rows (src/align.rs:105-192);
 *   - gap costs: a gap of length L costs open + (L-1)*extend (src/align.rs:198-223);
 *   - every score is the exact optimal Smith-Waterman-Gotoh local score, equal
 *     bit for bit to the reference's scalar i32 kernel (src/simd.rs:342-390).
 *
 * Threading: a context may be used from several host threads; calls on one
 * context are serialised internally.  Use one context per thread (each with
 * its own stream) for concurrent submission.
 */
#ifndef SABERTOOTH_B200_H
#define SABERTOOTH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ST_OK 0
#define ST_EINVAL -1    /* bad argument (null pointer, unknown id, size out of range) */
#define ST_ECUDA -2     /* CUDA runtime error */
#define ST_ENOMEM -3    /* device memory budget exceeded or allocation failure */
#define ST_ETIMEOUT -4  /* a bounded device wait expired (error status, context stays usable) */
#define ST_ESTATE -5    /* call order error (e.g. no database uploaded) */

/* Which kernel produced a score (src/simd.rs:40-49 Kernel, extended). */
#define ST_KERNEL_NONE 0     /* empty query or target: score 0 without a launch */
#define ST_KERNEL_GPU16 1    /* packed 16-bit DPX kernel, exact (no cell above the headroom) */
#define ST_KERNEL_GPU32 2    /* exact 32-bit kernel: rescore after 16-bit headroom, wide rows, gaps outside the 16-bit range, or band */

typedef struct st_ctx st_ctx;

/* ---- context ------------------------------------------------------------ */
/* hbm_budget_bytes = 0: no budget.  Replaces the rayon worker scratch set-up
 * (src/search.rs:708-712, SimdScratch src/simd.rs:142-156). */
st_ctx* st_init(int device, size_t hbm_budget_bytes);
void st_shutdown(st_ctx* ctx);
const char* st_last_error(void);
/* Launch everything of this context on a caller-owned cudaStream_t (NULL = the context's own stream). */
int st_set_stream(st_ctx* ctx, void* cuda_stream);
int st_synchronize(st_ctx* ctx);
/* Bytes of device memory the context holds. */
int st_mem_used(st_ctx* ctx, uint64_t* bytes);

/* ---- device-resident target database ----------------------------------- */
/* Residue arena + offsets, the layout of SeedIndex::seq/all_residues
 * (src/index.rs:1975-1979, 2324-2334) and SeqDb (src/fasta.rs).
 * offsets has n_seqs+1 entries; sequence s is residues[offsets[s] .. offsets[s+1]). */
int st_db_upload(st_ctx* ctx, const uint8_t* residues, const uint64_t* offsets, uint32_t n_seqs);
int st_db_info(st_ctx* ctx, uint32_t* n_seqs, uint64_t* n_residues);

/* ---- query profiles ----------------------------------------------------- */
/* QueryProfile::from_rows (src/simd.rs:172-210) / DiagProfile::build (src/ungapped.rs:214-255):
 * rows = int32 [m][21].  m = 0 is allowed (every score is then 0). */
int st_profile_create(st_ctx* ctx, const int32_t* rows, uint32_t m, uint32_t* id);
int st_profile_free(st_ctx* ctx, uint32_t id);
/* Batch form of st_profile_free (no reference counterpart: the reference drops
 * each QueryProfile on its own). Stops at the first unknown id, with the ids
 * before it freed. A freed id may be handed out again by a later create. */
int st_profiles_free(st_ctx* ctx, const uint32_t* ids, uint32_t n);
/* Batch form: n_profiles profiles from one rows arena; row_offsets[k]..row_offsets[k+1]
 * are the rows of profile k; ids written to ids[0..n_profiles).  Returns once
 * the rows are on the device (they may be reused); the device layouts are built
 * on the context's stream, before any later work that uses them.  The rows of a
 * profile whose scores all fit int8 travel to the device as int8. */
int st_profiles_create(st_ctx* ctx, const int32_t* rows, const uint64_t* row_offsets, uint32_t n_profiles,
                       uint32_t* ids);

/* ---- (G) Smith-Waterman-Gotoh score -------------------------------------- */
/* Plain per-call drop-in for QueryProfile::sw_score_with (src/simd.rs:252-292)
 * and sw_score (src/simd.rs:245): one host target, blocking (one upload, the
 * packed 16-bit kernel and the exact 32-bit one on the calling thread's call
 * slot). Safe to call from many host threads at once on one context: calls
 * run side by side on their own streams. kernel may be NULL. */
int st_sw_score(st_ctx* ctx, uint32_t profile, const uint8_t* target, uint32_t n, int32_t open, int32_t ext,
                int32_t* score, uint32_t* kernel);

/* One alignment task of the batched form: profile id, database ordinal and an
 * optional heuristic band (local_align_in_band, src/align.rs:954-970 with the
 * band rule of src/align.rs:439-447): band_radius < 0 = full local alignment,
 * else only cells with |j - i - band_center| <= band_radius (1-based i, j). */
typedef struct {
  uint32_t profile;
  uint32_t target;
  int32_t band_center;
  int32_t band_radius;
} st_pair;

/* Batched scoring of many (profile, database target) pairs with host buffers:
 * copies pairs in and scores out, plans (a tile class per query; on the GPU
 * for large batches), runs the persistent kernels and waits.  Replaces the
 * per-candidate loop Engine::search_query::score_one (src/search.rs:534-577).
 * kernels may be NULL. */
int st_sw_score_pairs(st_ctx* ctx, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext, int32_t* scores,
                      uint32_t* kernels);

/* The same in two halves, so that a caller can prepare the next batch (build
 * its profiles, fill its pairs) while this one runs on the GPU.
 * st_sw_score_pairs_async validates, uploads, plans and launches, then returns;
 * pairs may be reused at once, scores/kernels must stay valid (and unread)
 * until st_batch_wait, which waits, writes them and releases the batch.  Errors
 * in the arguments are reported by the first call; every batch must be waited
 * for.  (No reference counterpart: the reference scores candidates inline.) */
typedef struct st_batch st_batch;
int st_sw_score_pairs_async(st_ctx* ctx, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext,
                            int32_t* scores, uint32_t* kernels, st_batch** batch);
int st_batch_wait(st_batch* batch);
/* 0 when the batch's results are ready (st_batch_wait will not block), 1 while it runs. */
int st_batch_query(st_batch* batch);

/* ---- serving: continuous batching of requests ------------------------------
 * (No reference counterpart: the reference scores a search's queries in one
 * rayon pass.)  A server owns a worker thread on one context.  A request is
 * one query, as int32 [m][21] rows, and n database targets to score it against
 * (band_center/band_radius may be NULL: full local alignment).  Requests are
 * batched in arrival order as they come, up to max_batch_pairs pairs per batch
 * and hbm_budget_bytes of device memory for the batches in flight (two: one
 * running while the next is built and launched).  Scores equal those of the
 * same request scored alone.  submit copies its inputs and returns at once;
 * wait blocks until the request is done and returns its scores (cap entries)
 * and its latency from submit to completion in milliseconds. */
typedef struct st_server st_server;
st_server* st_server_create(st_ctx* ctx, int32_t open, int32_t ext, uint64_t max_batch_pairs,
                            uint64_t hbm_budget_bytes);
int st_server_submit(st_server* server, const int32_t* rows, uint32_t m, const uint32_t* targets,
                     const int32_t* band_center, const int32_t* band_radius, uint32_t n, uint64_t* request_id);
/* Many requests arriving together (one call, one lock): request k has rows
 * [row_offsets[k], row_offsets[k+1]) of rows and targets [target_offsets[k],
 * target_offsets[k+1]) of targets/band_center/band_radius; ids to request_ids[k]. */
int st_server_submit_many(st_server* server, uint32_t n_requests, const int32_t* rows, const uint64_t* row_offsets,
                          const uint32_t* targets, const uint64_t* target_offsets, const int32_t* band_center,
                          const int32_t* band_radius, uint64_t* request_ids);
int st_server_wait(st_server* server, uint64_t request_id, int32_t* scores, uint32_t cap, double* latency_ms);
int st_server_stats(st_server* server, uint64_t* batches, uint64_t* pairs);
void st_server_destroy(st_server* server);

/* Planned form over device buffers: a plan binds a pair list (copied at plan
 * time), gap costs and device output buffers; st_plan_run replays the captured
 * CUDA graph (asynchronous on the context stream). */
typedef struct st_plan st_plan;
int st_plan_create(st_ctx* ctx, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext, int32_t* d_scores,
                   uint32_t* d_kernels, st_plan** plan);
int st_plan_run(st_plan* plan);
int st_plan_stats(st_plan* plan, uint64_t* cells, uint64_t* rescored_pairs, uint32_t* n_launch_classes);
/* Runs each launch of the plan alone, timed with CUDA events on the context stream:
 * entry i = tile class index (-1 = the 32-bit kernel, -2 = the packed kernel of
 * banded pairs, whose cells are counted in the 32-bit entry), its planned cells
 * and its time.  cap >= n_launch_classes + 2; *n_out receives the count.  Scores
 * are written as by a run. */
int st_plan_profile(st_plan* plan, uint32_t cap, int32_t* classes, uint64_t* cells, float* ms, uint32_t* n_out);
void st_plan_destroy(st_plan* plan);

/* ---- (U) ungapped diagonal scoring --------------------------------------- */
/* One diagonal of score_batch (src/ungapped.rs:265-270 Lane): database
 * ordinal, diagonal d = target_pos - query_pos, query positions [lo, hi)
 * inside diag_range (src/ungapped.rs:38-46). */
typedef struct {
  uint32_t target;
  uint32_t lo;
  uint32_t hi;
  int32_t diag;
} st_lane;

/* Drop-in for ungapped::score_batch (src/ungapped.rs:285-386): out[i] =
 * kadane_score (src/ungapped.rs:53-62) of lanes[i] against the profile.  Host
 * buffers, blocking; any number of lanes per call. */
int st_ungapped_score(st_ctx* ctx, uint32_t profile, const st_lane* lanes, uint32_t n, int32_t* out);

/* The reference's Lane (src/ungapped.rs:265-270) field for field: `target` is
 * a slice (pointer + length) of the host residue arena that was given to
 * st_db_upload (the reference builds it from index.seq(tid),
 * src/prefilter.rs:1563-1568); diag and the query window [lo, hi) are as in
 * Lane.  Any slice of one database sequence is accepted. */
typedef struct {
  const uint8_t* target;
  uint64_t len;
  int64_t diag;
  uint64_t lo;
  uint64_t hi;
} st_lane_slice;

/* Drop-in for ungapped::score_batch (src/ungapped.rs:285-386) taking the
 * reference's lanes unchanged: out[i] = kadane_score of lanes[i].  A lane
 * whose slice is not inside the uploaded arena, or whose window is outside
 * diag_range of the slice, fails with ST_EINVAL.  Host buffers, blocking. */
int st_ungapped_score_slices(st_ctx* ctx, uint32_t profile, const st_lane_slice* lanes, uint32_t n, int32_t* out);

/* A prefilter seed hit: query profile id, database ordinal, diagonal.  The
 * scored window is the whole diagonal (diag_range; diag_window = 0 semantics). */
typedef struct {
  uint32_t query;
  uint32_t target;
  int32_t diag;
} st_hit;

/* Batched hits (the score_and_gate stage, src/prefilter.rs:1498-1660) with
 * host buffers: per_hit[i] = best ungapped segment score of hit i;
 * pair_best / pair_query / pair_target (capacity n) receive one entry per run
 * of consecutive hits with the same (query, target), in hit order, and
 * *n_pairs their count.  pair_* may be NULL to skip the per-pair output. */
int st_ungapped_hits(st_ctx* ctx, const st_hit* hits, uint64_t n, int32_t* per_hit, int32_t* pair_best,
                     uint32_t* pair_query, uint32_t* pair_target, uint64_t* n_pairs);
/* Same over device buffers, asynchronous on the context stream (d_n_pairs is a device uint64). */
int st_ungapped_hits_device(st_ctx* ctx, const st_hit* d_hits, uint64_t n, int32_t* d_per_hit,
                            int32_t* d_pair_best, uint32_t* d_pair_query, uint32_t* d_pair_target,
                            uint64_t* d_n_pairs);

/* ---- prefilter evidence, chain and gate -----------------------------------
 * The segment-evidence stage of prefilter_query (xdrop = 0, the default) for
 * the seed hits of many queries in one call: evaluate_block_kadane and
 * score_and_gate (src/prefilter.rs:1412-1660) followed by the candidate ranking
 * (:1074-1083).  Per (query, target): targets with fewer than min_hits hits are
 * dropped; the max_diagonals diagonals with the most hits (top_diagonals
 * :1194-1225, at most 16 scored) must include one with diag_hits hits; each is
 * scored by its best ungapped segment (kadane_segment, src/ungapped.rs:69-88)
 * over [qmin - diag_window, qmax + span + diag_window) clipped to diag_range
 * (the whole diagonal when diag_window = 0); the target's score is the best
 * segment or the best chain of two co-linear segments, sx + sy - gap(|dy - dx|)
 * (GapCosts::cost, src/align.rs:216-222), and it passes when the score is at
 * least min_diag_score. */

/* A seed hit: query profile id, database ordinal, diagonal = target position -
 * query position, query position (the reference's packed hit key,
 * src/prefilter.rs:1021-1036). */
typedef struct {
  uint32_t query;
  uint32_t target;
  int32_t diag;
  uint32_t qpos;
} st_seed_hit;

/* The evidence fields of PrefilterParams (src/prefilter.rs:262-303) plus the
 * seed span and the gap costs. */
typedef struct {
  uint32_t min_hits;
  uint32_t diag_hits;       /* >= 1 */
  uint32_t max_diagonals;   /* >= 1 */
  uint32_t diag_window;     /* 0 = whole diagonal */
  uint32_t span;            /* seed pattern span (k for contiguous seeds) */
  int32_t min_diag_score;
  int32_t gap_open;
  int32_t gap_ext;
  uint32_t max_candidates;  /* per query, 0 = all */
  uint32_t regions;         /* 1 = compute t_lo..t_hi, 0 = report 0..UINT32_MAX */
} st_prefilter_params;

/* Candidate (src/prefilter.rs:370-381) plus its query id. */
typedef struct {
  uint32_t query;
  uint32_t target;
  uint32_t hits;
  int32_t diag_score;
  int64_t best_diag;
  uint32_t t_lo;
  uint32_t t_hi;
} st_candidate;

/* The evidence counters of PrefilterStats, summed over the call's queries,
 * plus hits_rejected: hits outside their query or target, or with an unknown
 * profile id (they are skipped and the call returns ST_EINVAL). */
typedef struct {
  uint64_t targets_hit;
  uint64_t targets_evaluated;
  uint64_t diagonals_scored;
  uint64_t chains_used;
  uint64_t candidates;
  uint64_t candidates_capped;
  uint64_t hits_rejected;
} st_prefilter_stats;

/* Host buffers.  Candidates are ordered by query id, then score descending,
 * then target ascending, at most max_candidates per query.  *n_out receives the
 * total; the first min(cap, total) are written to out (cap = n always
 * suffices).  stats may be NULL.  Fewer than 2^31 - 1 hits per call. */
int st_prefilter_gate(st_ctx* ctx, const st_seed_hit* hits, uint64_t n, const st_prefilter_params* params,
                      st_candidate* out, uint64_t cap, uint64_t* n_out, st_prefilter_stats* stats);
/* Device buffers (d_out has room for n candidates); n_out and stats are host
 * pointers.  Returns once the candidates are written (it reads the candidate
 * count from the device to size the ranking). */
int st_prefilter_gate_device(st_ctx* ctx, const st_seed_hit* d_hits, uint64_t n, const st_prefilter_params* params,
                             st_candidate* d_out, uint64_t* n_out, st_prefilter_stats* stats);

/* ---- seed hits ---------------------------------------------------------------
 * The seed stage of prefilter_query (src/prefilter.rs:816-995) on the device.
 * st_seed_index_build indexes the uploaded database for a seed pattern given
 * as a 0/1 mask that starts and ends with '1' (SeedPattern::from_mask,
 * src/prefilter.rs:101-124; weight 2..7 here): every window whose care
 * residues are all standard (codes < 20), keyed by those residues in base 20
 * (the seeding pass of src/index.rs:1059-1074).  An upload of a new database
 * drops the index. */
int st_seed_index_build(st_ctx* ctx, const char* seed_mask);

/* The similar-k-mer fields of PrefilterParams (src/prefilter.rs:262-303). */
typedef struct {
  int32_t kmer_score;          /* threshold of a similar k-mer's summed score */
  uint32_t max_kmers_per_pos;  /* >= 1: the first this many k-mers of the canonical order per window */
  uint32_t exact_seeds;        /* add the query's own k-mer (sequence queries) */
  uint32_t max_seed_occ;       /* skip k-mers with more postings (0 = never) */
} st_seed_params;

/* The seed counters of PrefilterStats, summed over the call's queries. */
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
} st_seed_stats;

/* Seed hits of n_queries queries (profile ids; seed rows = the profiles' rows).
 * residues (optional) holds each sequence query's residue codes,
 * residues[residue_offsets[i] .. residue_offsets[i+1]) with one code per
 * profile row: windows with a care residue >= 20 are skipped and, with
 * exact_seeds, the query's own k-mer is added; NULL for profile (PSSM) queries.
 * Per window (every start in [0, m - span]): the first max_kmers_per_pos
 * k-mers scoring >= kmer_score in the canonical order (score descending, then
 * the rank vector ascending: top_kmers, src/prefilter.rs:457-568), then one hit
 * per posting.  *n_out receives the hit count; the first min(cap, count) hits
 * are written, in no particular order.  Windows whose rows span more than 1,024
 * score values above the threshold are rejected (ST_EINVAL). */
int st_seed_hits(st_ctx* ctx, const uint32_t* profiles, uint32_t n_queries, const uint8_t* residues,
                 const uint64_t* residue_offsets, const st_seed_params* params, st_seed_hit* out, uint64_t cap,
                 uint64_t* n_out, st_seed_stats* stats);

/* The whole prefilter of prefilter_query for a batch of queries on the device:
 * seed hits (as st_seed_hits) -> evidence, chains and gate -> ranked
 * candidates (as st_prefilter_gate; params->span is taken from the index's
 * pattern).  The profile ids of one call must be distinct.  Host buffers; stats
 * and seed_stats may be NULL. */
int st_prefilter_queries(st_ctx* ctx, const uint32_t* profiles, uint32_t n_queries, const uint8_t* residues,
                         const uint64_t* residue_offsets, const st_seed_params* seed_params,
                         const st_prefilter_params* params, st_candidate* out, uint64_t cap, uint64_t* n_out,
                         st_prefilter_stats* stats, st_seed_stats* seed_stats);

/* ---- search serving ------------------------------------------------------------
 * (No reference counterpart: the reference runs a search's queries in one rayon
 * pass.)  A search server owns a worker thread on one context whose database
 * has a seed index.  A request is one bare query — its int32 [m][21] rows and,
 * for sequence queries (sequence_queries = 1), its m residue codes.  The worker
 * takes every request that has arrived (up to max_batch_queries, 0 = 4,096)
 * as one batch and runs the whole search for it: st_prefilter_queries, then
 * the exact SW score of every candidate (gaps from params); requests that
 * arrive meanwhile form the next batch.  Results equal those of the query
 * searched alone.  wait returns the request's candidates (query field 0,
 * ranked as by st_prefilter_queries) with their SW scores and its latency from
 * submit to completion in milliseconds; with cap below the count it only sets
 * *n_out and the request can be waited for again. */
typedef struct st_search_server st_search_server;
st_search_server* st_search_server_create(st_ctx* ctx, const st_seed_params* seed_params,
                                          const st_prefilter_params* params, int sequence_queries,
                                          uint32_t max_batch_queries);
int st_search_server_submit(st_search_server* s, const int32_t* rows, uint32_t m, const uint8_t* residues,
                            uint64_t* request_id);
int st_search_server_wait(st_search_server* s, uint64_t request_id, st_candidate* candidates, int32_t* scores,
                          uint64_t cap, uint64_t* n_out, double* latency_ms);
int st_search_server_stats(st_search_server* s, uint64_t* batches, uint64_t* queries);
void st_search_server_destroy(st_search_server* s);

/* ---- per-profile calibration ----------------------------------------------
 * calibrate_profile (src/evalue.rs:714-748) for many profiles at once: sample i
 * (0 <= i < samples) is a background target drawn from the SplitMix64 stream
 * stream_seed(seed, 0xBEEF, i) (src/evalue.rs:53-81): length
 * lengths[below(n_lengths)] (at least 1), residues from BackgroundSampler
 * (:84-114) over p_back (the 20 standard background probabilities of the
 * matrix).  Every profile is scored against every sample (exact SW-Gotoh, the
 * batched path; the targets are generated on the device and replace the
 * database for this call only), then a Gumbel is fitted by maximum likelihood
 * (fit_gumbel_ml, :138-182) and K = exp(lambda (mu + 1/2)) / (m * mean length).
 * The reference calls it per PSSM with the search's seed (0x5EED) and a sample
 * of database lengths (src/search.rs:467-481), so all profiles of a search
 * share the same targets.  out[p].ok = 0 where the reference returns None
 * (no lengths, an empty profile, fewer than 10 samples, a degenerate fit).
 * scores may be NULL, else [n_profiles][samples]. */
typedef struct {
  double lambda;
  double k;
  double mu;
  uint32_t n;  /* samples */
  int32_t ok;
} st_calibration;
int st_calibrate_profiles(st_ctx* ctx, const uint32_t* profiles, uint32_t n_profiles, const uint32_t* lengths,
                          uint32_t n_lengths, uint32_t samples, uint64_t seed, const double* p_back, int32_t open,
                          int32_t ext, int32_t* scores, st_calibration* out);

/* ---- end cells and alignment spans ---------------------------------------
 * Score plus end cell, the first optimum in column-major order (smallest target
 * position, then smallest query position): QueryProfile::sw_score_end_with
 * (src/simd.rs:301-326, tie rule :375-381).  Positions are 0-based and
 * inclusive; -1 when the score is 0 (the reference returns None).  Computed by
 * the exact 32-bit kernel.  Unbanded pairs only. */
int st_sw_score_end(st_ctx* ctx, uint32_t profile, const uint8_t* target, uint32_t n, int32_t open, int32_t ext,
                    int32_t* score, int32_t* q_end, int32_t* t_end);
/* Batched: ends[2i], ends[2i+1] = (query end, target end) of pair i. */
int st_sw_score_end_pairs(st_ctx* ctx, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext, int32_t* scores,
                          int32_t* ends);
/* End cell plus start cell of each pair's alignment: the two score passes of
 * align_canonical (src/align.rs:848-866): the forward end pass, then the same
 * pass over the query rows [0, q_end] and target [0, t_end], both reversed,
 * whose end cell (a, b) gives the start (q_end - a, t_end - b).
 * starts[2i], starts[2i+1] = (query start, target start). */
int st_sw_align_span_pairs(st_ctx* ctx, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext,
                           int32_t* scores, int32_t* ends, int32_t* starts);

/* ---- tile classes and autotuning ----------------------------------------- */
/* The packed 16-bit kernel runs in tile classes: G lanes per alignment x R
 * query rows per lane x C target columns per wavefront step.  In a batch each
 * query takes the class with the least estimated time: its streamed cells
 * (padded rows x padded columns) over the class's rate (streamed cells per
 * second / 1e12; built-in B200 figures until st_autotune measures them; a rate
 * of 0 leaves the class out).  A per-context table maps (query-length bin,
 * mean target-length bin) to a class that is then forced; -1 entries (the
 * default) use the rates.  Query bins: <=32, <=64, ..., <=8192, >8192 (10);
 * target bins: <=64, <=128, ..., <=4096, >4096 (8); the table is row-major
 * [10][8].  (No reference counterpart: the reference picks SIMD widths at run
 * time, src/simd.rs:59-124.) */
int st_tune_num_classes(void);
int st_tune_class_shape(int cls, int* lanes_per_alignment, int* rows_per_lane, int* cols_per_step);
int st_tune_get(st_ctx* ctx, int32_t* table);
int st_tune_set(st_ctx* ctx, const int32_t* table);
/* Per-class rates: rates[k] for k < min(cap, st_tune_num_classes()). */
int st_tune_get_rates(st_ctx* ctx, float* rates, uint32_t cap);
int st_tune_set_rates(st_ctx* ctx, const float* rates, uint32_t n);
/* Measures every class's rate on a sample of the pairs (whole queries, spread
 * over the batch, up to max_pairs pairs) by planning it with all queries forced
 * into that class; the forcing table is left as it was. */
int st_autotune(st_ctx* ctx, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext,
                uint32_t max_pairs, uint32_t* classes_calibrated);

/* ---- allocation-free scoring ----------------------------------------------- */
/* Exact SW-Gotoh score of ONE pair over caller-owned device buffers, with no
 * device memory allocation: for callers that cannot call cudaMalloc/cudaFree
 * (code running inside a global-mode stream capture, latency-bound serving
 * threads that cannot take the implicit synchronisation of cudaFree, processes
 * whose device memory belongs to another allocator's pool).  No counterpart in
 * the reference: it is an addition of this library.
 *   d_rows:   device int32 [m][21] score rows (the ScoreTable layout), m <= 2^20
 *   d_target: device residue codes, n <= 65536 (longer targets: ST_EINVAL)
 *   d_score:  device int32 receiving the score (0 when m or n is 0)
 * Asynchronous on `stream` (a cudaStream_t, NULL = legacy default stream).  The
 * kernel's scratch is a fixed 512 KiB static device array that every GPU
 * loading the library holds until exit; all calls on a device share it, so
 * calls that overlap on the GPU race and must be ordered by the caller.  The
 * first call on a device resolves the array's address and keeps it for the
 * process; make it before any stream capture.  A cudaDeviceReset discards the
 * device's copy of the array, so the kept address is stale afterwards: reset
 * no device that this entry point has run on.  Nothing in the array needs to
 * start at zero (a call writes every boundary entry before it reads it back).
 * Same scores as st_sw_score for every gap cost. */
int st_sw_score_noalloc(const int32_t* d_rows, uint32_t m, const uint8_t* d_target, uint32_t n, int32_t open,
                        int32_t ext, int32_t* d_score, void* stream);

/* ---- measurement helpers -------------------------------------------------- */
/* Device-wide throughput of the packed s16x2 DPX add-max instruction
 * (__viaddmax_s16x2), in lane-operations per second, measured on the current
 * device with CUDA events (the denominator of the SW roofline). */
int st_probe_dpx(st_ctx* ctx, double* ops_per_s);
/* Number of kernel launches this context issued since creation. */
int st_launch_count(st_ctx* ctx, uint64_t* launches);

#ifdef __cplusplus
}
#endif
#endif
