// Packed 16-bit Smith-Waterman-Gotoh score kernel (the fast path of the
// reference's QueryProfile::sw_score_with, src/simd.rs:252-292).
//
// Layout of the work: a group of G lanes of one warp scores TWO targets of the
// same query at once, one per 16-bit half of every register (s16x2).  Lane l of
// the group owns R consecutive query rows; the target streams through the
// group one column per step as a wavefront (lane l works on column c while
// lane l-1 works on column c+1), so the bottom-row H and the F entering the
// next lane travel by one __shfl_up_sync per step.  Queries longer than G*R
// rows are scored in passes over the target; the bottom row of a pass (H and
// F per column) is kept in a global scratch line per group, which lane 0 of
// the next pass reads back.  Passes follow each other without draining the
// wavefront.
//
// Recurrence per cell (literally Gotoh's, as the reference's scalar kernel
// src/simd.rs:361-374):
//   H = max(Hdiag + S, E, F, 0)
//   E' = max(E - extend, H - open)        (E of the next column)
//   F' = max(F - extend, H - open)        (F of the next row)
// with DPX ops: t = viaddmax(Hdiag, S, E); H = vimax_relu(t, F);
// Ho = vadd2(H, -open); E' = viaddmax(E, -ext, Ho); F' = viaddmax(F, -ext, Ho).
//
// Exactness: the adds wrap instead of saturating.  If no H anywhere exceeds
// T = 32767 - max(0, max score), no sum can leave the int16 range (E, F >=
// -open-extend, S is int8), so the result is exact; otherwise the first H
// above T was itself computed exactly and the pair is flagged for the exact
// 32-bit kernel.  Rows past the query and columns past a target score 0, which
// cannot raise the maximum when open, extend >= 0 (the only gap costs this
// kernel is used for).
#pragma once
#include "st_common.cuh"

namespace st {

struct Sw16CtaTask {
  uint32_t query;
  uint32_t wt_begin;
  uint32_t wt_end;
  uint32_t m_pad;  // P * G * R rows staged in shared memory
};

struct Sw16WarpTask {
  uint32_t slot_begin;  // 64/G consecutive entries of slot_pair
  uint32_t ncols;       // columns streamed per pass: multiple of 16, >= 32
};

struct Sw16Params {
  DeviceDb db;
  DeviceProfiles prof;
  const Sw16CtaTask* cta_tasks;
  uint32_t n_cta_tasks;
  const Sw16WarpTask* warp_tasks;
  const uint32_t* slot_pair;    // pair index or kNoPair
  const uint32_t* pair_target;  // database ordinal of pair p
  int32_t* scores;              // per pair
  uint32_t* kernels;            // per pair (may be null)
  uint32_t* ovf_count;          // pairs above the 16-bit headroom
  uint32_t* ovf_pairs;
  uint32_t* work_counter;       // next CTA task (zeroed before each launch)
  uint2* scratch;               // pass boundary rows, scratch_stride per group
  uint32_t scratch_stride;
  int32_t open, ext;
};

constexpr uint32_t kNoPair = 0xFFFFFFFFu;

template <int G, int R>
struct Sw16Tile {
  static_assert(G == 4 || G == 8 || G == 16 || G == 32, "group size");
  static_assert(R == 8 || R == 16 || R == 32, "rows per lane");
  static constexpr int kGroupsPerWarp = 32 / G;
  static constexpr int kSlots = 2 * kGroupsPerWarp;
  static constexpr int kWords = R / 4;
};

// Loads this lane's R profile bytes of one residue row (R/4 words).
template <int R>
__device__ __forceinline__ void load_rows8(const int8_t* p, uint32_t (&w)[R / 4]) {
  if constexpr (R % 16 == 0) {
#pragma unroll
    for (int v = 0; v < R / 16; ++v) {
      uint4 x = *reinterpret_cast<const uint4*>(p + 16 * v);
      w[4 * v + 0] = x.x;
      w[4 * v + 1] = x.y;
      w[4 * v + 2] = x.z;
      w[4 * v + 3] = x.w;
    }
  } else {
    uint2 x = *reinterpret_cast<const uint2*>(p);
    w[0] = x.x;
    w[1] = x.y;
  }
}

template <int G, int R>
__device__ __forceinline__ void sw16_warp_task(const Sw16Params& prm, const int8_t* __restrict__ prof_s,
                                               uint32_t m_pad, uint32_t P, int32_t thresh,
                                               const Sw16WarpTask& wt, uint32_t group_id) {
  using Tile = Sw16Tile<G, R>;
  const int lane = threadIdx.x & 31;
  const int gl = lane % G;
  const int grp = lane / G;
  const uint32_t FULL = 0xFFFFFFFFu;

  // the two targets of this group
  const uint32_t pA = prm.slot_pair[wt.slot_begin + 2 * grp];
  const uint32_t pB = prm.slot_pair[wt.slot_begin + 2 * grp + 1];
  const uint8_t* tA = nullptr;
  const uint8_t* tB = nullptr;
  uint32_t lenA = 0, lenB = 0;  // readable bytes (padded to 16)
  if (pA != kNoPair) {
    uint32_t t = prm.pair_target[pA];
    tA = prm.db.arena + prm.db.offset[t];
    lenA = (prm.db.length[t] + 15u) & ~15u;
  }
  if (pB != kNoPair) {
    uint32_t t = prm.pair_target[pB];
    tB = prm.db.arena + prm.db.offset[t];
    lenB = (prm.db.length[t] + 15u) & ~15u;
  }
  const int ncols = static_cast<int>(wt.ncols);
  const uint32_t MOPEN = pk_splat(-prm.open);
  const uint32_t MEXT = pk_splat(-prm.ext);
  const uint32_t E0 = MOPEN;  // E of the first column: max(0 - open, -inf)
  const uint32_t F0 = MOPEN;  // F of the first row
  const uint32_t SENT2 = kSentinel | (kSentinel << 8);

  uint32_t Hp[R], E[R];
#pragma unroll
  for (int k = 0; k < R; ++k) {
    Hp[k] = 0;
    E[k] = E0;
  }
  uint32_t best = 0, hup_prev = 0, h_bot = 0, f_out = F0, res = SENT2;
  int c = -gl;  // this lane's column; negative = not started yet
  uint32_t pass = 0;
  uint2* bnd = prm.scratch + static_cast<size_t>(group_id) * prm.scratch_stride;

  // lane 0 streams residues one column ahead
  uint32_t nxt = SENT2;
  if (gl == 0) {
    uint32_t a = (0 < static_cast<int>(lenA)) ? __ldg(tA) : kSentinel;
    uint32_t b = (0 < static_cast<int>(lenB)) ? __ldg(tB) : kSentinel;
    nxt = min(a, static_cast<uint32_t>(kSentinel)) | (min(b, static_cast<uint32_t>(kSentinel)) << 8);
  }

  const int steps = static_cast<int>(P) * ncols + G - 1;
  const int lane_row0 = gl * R;
  const int rows_per_pass = G * R;

  for (int s = 0; s < steps; ++s) {
    uint32_t hin = __shfl_up_sync(FULL, h_bot, 1, G);
    uint32_t fin = __shfl_up_sync(FULL, f_out, 1, G);
    uint32_t rin = __shfl_up_sync(FULL, res, 1, G);
    if (gl == 0) {
      if (pass < P) {
        rin = nxt;
        // prefetch the residues of the next column (next pass wraps to column 0)
        int cn = c + 1;
        bool last = (cn == ncols);
        if (last) cn = 0;
        if (last && pass + 1 >= P) {
          nxt = SENT2;
        } else {
          uint32_t a = (cn < static_cast<int>(lenA)) ? __ldg(tA + cn) : kSentinel;
          uint32_t b = (cn < static_cast<int>(lenB)) ? __ldg(tB + cn) : kSentinel;
          nxt = min(a, static_cast<uint32_t>(kSentinel)) | (min(b, static_cast<uint32_t>(kSentinel)) << 8);
        }
        if (pass > 0) {
          uint2 bv = bnd[c];
          hin = bv.x;
          fin = bv.y;
        } else {
          hin = 0;
          fin = F0;
        }
      } else {
        rin = SENT2;
        hin = 0;
        fin = F0;
      }
    }
    res = rin;
    if (c == 0) {  // first column of a pass: left border H = 0, E = first-column E
#pragma unroll
      for (int k = 0; k < R; ++k) {
        Hp[k] = 0;
        E[k] = E0;
      }
      hup_prev = 0;
    }
    const uint32_t pp = pass < P ? pass : P - 1;
    const int8_t* rowA = prof_s + (res & 0xFFu) * m_pad + pp * rows_per_pass + lane_row0;
    const int8_t* rowB = prof_s + (res >> 8) * m_pad + pp * rows_per_pass + lane_row0;
    uint32_t wa[Tile::kWords], wb[Tile::kWords];
    load_rows8<R>(rowA, wa);
    load_rows8<R>(rowB, wb);

    uint32_t hd = hup_prev;
    uint32_t F = fin;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const uint32_t S = prmt(wa[k >> 2], wb[k >> 2], sel_pair(k & 3));
      const uint32_t t = pk_addmax(hd, S, E[k]);
      const uint32_t H = pk_max_relu(t, F);
      best = pk_max(best, H);
      const uint32_t Ho = pk_add(H, MOPEN);
      E[k] = pk_addmax(E[k], MEXT, Ho);
      F = pk_addmax(F, MEXT, Ho);
      hd = Hp[k];
      Hp[k] = H;
    }
    hup_prev = hin;
    h_bot = Hp[R - 1];
    f_out = F;
    if (gl == G - 1 && pass + 1 < P && c >= 0) bnd[c] = make_uint2(h_bot, f_out);
    if (++c == ncols) {
      c = 0;
      ++pass;
    }
    __syncwarp();
  }

  // group maximum
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) best = pk_max(best, __shfl_xor_sync(FULL, best, o, G));
  if (gl == 0) {
    const int32_t bA = pk_lo(best), bB = pk_hi(best);
    if (pA != kNoPair) {
      if (bA > thresh) {
        prm.ovf_pairs[atomicAdd(prm.ovf_count, 1u)] = pA;
      } else {
        prm.scores[pA] = bA;
        if (prm.kernels) prm.kernels[pA] = 1u;
      }
    }
    if (pB != kNoPair) {
      if (bB > thresh) {
        prm.ovf_pairs[atomicAdd(prm.ovf_count, 1u)] = pB;
      } else {
        prm.scores[pB] = bB;
        if (prm.kernels) prm.kernels[pB] = 1u;
      }
    }
  }
}

// Persistent kernel: CTAs pull CTA tasks (one query each) from a global
// counter, stage that query's int8 profile in shared memory, and their warps
// pull warp tasks of the CTA task from a shared counter.
template <int G, int R, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) sw16_kernel(const Sw16Params prm) {
  extern __shared__ __align__(16) int8_t prof_s[];
  __shared__ uint32_t s_task, s_next;
  using Tile = Sw16Tile<G, R>;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t group_base = (blockIdx.x * WARPS + warp) * Tile::kGroupsPerWarp;
  const uint32_t group_id = group_base + lane / G;

  for (;;) {
    if (threadIdx.x == 0) s_task = atomicAdd(prm.work_counter, 1u);
    __syncthreads();
    const uint32_t ct = s_task;
    if (ct >= prm.n_cta_tasks) break;
    const Sw16CtaTask task = prm.cta_tasks[ct];
    const uint32_t q = task.query;
    const uint32_t m_pad = task.m_pad;
    const uint32_t P = m_pad / (G * R);
    // stage the profile: 22 residue rows of m_pad int8 scores, zero past the stored stride
    {
      const uint32_t chunks_per_row = m_pad / 16;
      const uint32_t stride = prm.prof.stride8[q];
      const int8_t* src = prm.prof.p8[q];
      for (uint32_t idx = threadIdx.x; idx < kProfRows * chunks_per_row; idx += WARPS * 32) {
        const uint32_t r = idx / chunks_per_row;
        const uint32_t i = (idx - r * chunks_per_row) * 16;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (i < stride) v = *reinterpret_cast<const uint4*>(src + static_cast<size_t>(r) * stride + i);
        *reinterpret_cast<uint4*>(prof_s + static_cast<size_t>(r) * m_pad + i) = v;
      }
    }
    if (threadIdx.x == 0) s_next = task.wt_begin;
    const int32_t thresh = 32767 - prm.prof.max_score[q];
    __syncthreads();
    for (;;) {
      uint32_t w = 0;
      if (lane == 0) w = atomicAdd(&s_next, 1u);
      w = __shfl_sync(0xFFFFFFFFu, w, 0);
      if (w >= task.wt_end) break;
      const Sw16WarpTask wt = prm.warp_tasks[w];
      sw16_warp_task<G, R>(prm, prof_s, m_pad, P, thresh, wt, group_id);
    }
    __syncthreads();
  }
}

}  // namespace st
