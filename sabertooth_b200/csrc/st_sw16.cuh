// Packed 16-bit Smith-Waterman-Gotoh score kernel (the fast path of the
// reference's QueryProfile::sw_score_with, src/simd.rs:252-292).
//
// Work layout.  A group of G lanes of one warp scores TWO targets of the same
// query at once, one per 16-bit half of every register (s16x2).  Lane l of the
// group owns R consecutive query rows; the targets stream through the group as
// a wavefront, C columns per step (lane l works on columns [c, c+C) while lane
// l-1 works on [c+C, c+2C)), so per step each lane receives from the lane
// above, by __shfl_up_sync, a control word, the residue codes of its C
// columns, and the bottom-row H and the F entering its first row for each of
// them.  Queries longer than G*R rows are scored in passes over the targets;
// the bottom row of a pass goes through a per-group scratch line in global
// memory and comes back into lane 0 for the next pass.
//
// Streaming.  A warp pulls warp tasks (64/G targets of the query, two per
// group, padded to a common length) one after another and feeds them into the
// wavefront back to back: lane 0 starts the next task while the lower lanes
// finish the previous one, so the G-1 step ramp is paid once per query, not
// per task.  The control word that travels with the columns tells each lane
// the column, the pass, when to reset its state (first column of a pass) and
// when a task ends; at that point every lane folds its running maximum into
// the task's slot in shared memory, and the last lane of the group, which
// finishes the task last, writes the two scores.  The next task is claimed and
// its slot records loaded one task ahead, so the loads are off the critical
// path.
//
// Recurrence per cell (literally Gotoh's, as the reference's scalar kernel
// src/simd.rs:361-374):
//   H = max(Hdiag + S, E, F, 0)
//   E' = max(E - extend, H - open)        (E of the next column)
//   F' = max(F - extend, H - open)        (F of the next row)
// with DPX ops: t = viaddmax(Hdiag, S, E); H = vimax_relu(t, F);
// Ho = vadd2(H, -open); E' = viaddmax(E, -ext, Ho); F' = viaddmax(F, -ext, Ho).
//
// Exactness.  The adds wrap instead of saturating.  If no H anywhere exceeds
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
  uint32_t slot_begin;  // 64/G consecutive slot records, two per group
  uint32_t ncols;       // columns streamed per pass: multiple of 4, >= 32 (>= C*G with several passes)
};

// One target of a warp task: everything lane 0 needs, in one 16-byte load.
struct Sw16Slot {
  uint32_t pair;    // pair index, kNoPair for an empty slot
  uint32_t toff16;  // database arena offset of the target / 16
  uint32_t tlen16;  // target length rounded up to 16 (readable bytes)
  uint32_t tlen;    // target length
};

struct Sw16Params {
  const uint8_t* arena;  // padded residue arena
  DeviceProfiles prof;
  const Sw16CtaTask* cta_tasks;
  uint32_t n_cta_tasks;
  const Sw16WarpTask* warp_tasks;
  const Sw16Slot* slots;
  int32_t* scores;        // per pair
  uint32_t* kernels;      // per pair (may be null)
  uint32_t* ovf_count;    // pairs above the 16-bit headroom
  uint32_t* ovf_pairs;
  uint32_t* work_counter; // next CTA task (reset before each launch)
  uint2* scratch;         // pass boundary rows, scratch_stride entries per group
  const uint2* zline;     // (H, F) = (0, first-row F) for every column: the input of a first pass
  uint32_t scratch_stride;
  int32_t open, ext;
};

constexpr uint32_t kNoPair = 0xFFFFFFFFu;

// control word: column (16 bits) | pass (8) | task slot (3) | last step of the task | idle
constexpr uint32_t kCtlLast = 1u << 27;
constexpr uint32_t kCtlIdle = 1u << 28;
constexpr int kSlotRing = 8;

template <int G, int R, int C>
struct Sw16Tile {
  static_assert(G == 4 || G == 8 || G == 16 || G == 32, "group size");
  static_assert(R % 4 == 0 && R >= 8 && R <= 32, "rows per lane");
  static_assert(C == 1 || C == 2 || C == 4, "columns per step");
  static constexpr int kGroups = 32 / G;
  static constexpr int kSlots = 2 * kGroups;
  static constexpr int kWords = R / 4;
};

// This lane's R profile bytes of one residue row (R/4 words); the lane's
// first row is R-byte aligned, so the widest vector that divides R is used.
template <int R>
__device__ __forceinline__ void load_rows8(const int8_t* p, uint32_t (&w)[R / 4]) {
  if constexpr (R % 16 == 0) {
#pragma unroll
    for (int v = 0; v < R / 16; ++v) {
      const uint4 x = *reinterpret_cast<const uint4*>(p + 16 * v);
      w[4 * v + 0] = x.x;
      w[4 * v + 1] = x.y;
      w[4 * v + 2] = x.z;
      w[4 * v + 3] = x.w;
    }
  } else if constexpr (R % 8 == 0) {
#pragma unroll
    for (int v = 0; v < R / 8; ++v) {
      const uint2 x = *reinterpret_cast<const uint2*>(p + 8 * v);
      w[2 * v + 0] = x.x;
      w[2 * v + 1] = x.y;
    }
  } else {
#pragma unroll
    for (int v = 0; v < R / 4; ++v) w[v] = *reinterpret_cast<const uint32_t*>(p + 4 * v);
  }
}

// C residue codes of a target starting at column c (c is a multiple of C), or sentinels past its end.
template <int C>
__device__ __forceinline__ uint32_t load_codes(const uint8_t* t, uint32_t len16, int c) {
  constexpr uint32_t sent = 0x15151515u & (C == 4 ? 0xFFFFFFFFu : (C == 2 ? 0xFFFFu : 0xFFu));
  if (static_cast<uint32_t>(c) >= len16) return sent;
  if constexpr (C == 4) return __ldg(reinterpret_cast<const uint32_t*>(t + c));
  else if constexpr (C == 2) return __ldg(reinterpret_cast<const uint16_t*>(t + c));
  else return __ldg(t + c);
}

template <int C>
__device__ __forceinline__ void load_bnd(const uint2* b, uint32_t (&h)[C], uint32_t (&f)[C]) {
  if constexpr (C == 4) {
    const uint4 x = *reinterpret_cast<const uint4*>(b);
    const uint4 y = *reinterpret_cast<const uint4*>(b + 2);
    h[0] = x.x; f[0] = x.y; h[1] = x.z; f[1] = x.w;
    h[2] = y.x; f[2] = y.y; h[3] = y.z; f[3] = y.w;
  } else if constexpr (C == 2) {
    const uint4 x = *reinterpret_cast<const uint4*>(b);
    h[0] = x.x; f[0] = x.y; h[1] = x.z; f[1] = x.w;
  } else {
    const uint2 x = *b;
    h[0] = x.x; f[0] = x.y;
  }
}

template <int C>
__device__ __forceinline__ void store_bnd(uint2* b, const uint32_t (&h)[C], const uint32_t (&f)[C]) {
  if constexpr (C == 4) {
    *reinterpret_cast<uint4*>(b) = make_uint4(h[0], f[0], h[1], f[1]);
    *reinterpret_cast<uint4*>(b + 2) = make_uint4(h[2], f[2], h[3], f[3]);
  } else if constexpr (C == 2) {
    *reinterpret_cast<uint4*>(b) = make_uint4(h[0], f[0], h[1], f[1]);
  } else {
    *b = make_uint2(h[0], f[0]);
  }
}

// Per-group view of a warp task's two targets (meaningful in the group's lane 0).
struct Sw16Pair2 {
  const uint8_t* tA;
  const uint8_t* tB;
  uint32_t lenA, lenB;
  uint32_t pA, pB;
};

__device__ __forceinline__ Sw16Pair2 load_pair2(const Sw16Params& prm, uint32_t slot_begin, int grp) {
  const uint4 a = __ldg(reinterpret_cast<const uint4*>(prm.slots + slot_begin + 2 * grp));
  const uint4 b = __ldg(reinterpret_cast<const uint4*>(prm.slots + slot_begin + 2 * grp + 1));
  Sw16Pair2 r;
  r.pA = a.x;
  r.pB = b.x;
  r.tA = prm.arena + static_cast<size_t>(a.y) * 16;
  r.tB = prm.arena + static_cast<size_t>(b.y) * 16;
  r.lenA = a.x == kNoPair ? 0u : a.z;
  r.lenB = b.x == kNoPair ? 0u : b.z;
  return r;
}

// Persistent kernel: CTAs pull CTA tasks (one query each) from a global
// counter and stage the query's int8 profile in shared memory; each warp then
// streams the CTA task's warp tasks, claimed from a shared counter.
template <int G, int R, int C, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) sw16_kernel(const Sw16Params prm) {
  using Tile = Sw16Tile<G, R, C>;
  constexpr int NG = Tile::kGroups;
  constexpr uint32_t FULL = 0xFFFFFFFFu;
  extern __shared__ __align__(16) int8_t prof_s[];
  __shared__ uint32_t s_task, s_next;
  __shared__ int32_t s_best[WARPS][NG][kSlotRing][2];
  __shared__ uint32_t s_pair[WARPS][NG][kSlotRing][2];

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int gl = lane % G;
  const int grp = lane / G;
  uint2* bnd = prm.scratch + static_cast<size_t>((blockIdx.x * WARPS + warp) * NG + grp) * prm.scratch_stride;
  const uint32_t MOPEN = pk_splat(-prm.open);
  const uint32_t MEXT = pk_splat(-prm.ext);
  const uint32_t E0 = MOPEN;  // E of the first column: max(0 - open, -inf)
  const uint32_t F0 = MOPEN;  // F of the first row
  const uint32_t SENTW = 0x15151515u;

  for (;;) {
    if (threadIdx.x == 0) s_task = atomicAdd(prm.work_counter, 1u);
    __syncthreads();
    const uint32_t ct = s_task;
    if (ct >= prm.n_cta_tasks) break;
    const Sw16CtaTask task = prm.cta_tasks[ct];
    const uint32_t q = task.query;
    const uint32_t m_pad = task.m_pad;
    const int P = static_cast<int>(m_pad / (G * R));
    {  // stage the profile: 22 residue rows of m_pad int8 scores, zero past the stored stride
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

    // ---- the warp's stream over warp tasks ----
    // The group's last lane (the feeder) tracks lane 0's position in the stream (the same
    // uniform state in every lane), loads the targets' residues and the previous pass's
    // bottom row for lane 0's next step, and leaves them in its outgoing registers: the
    // rotating shuffle then hands lane 0 the stream and every other lane its upper
    // neighbour's outputs.
    const bool feeder = gl == G - 1;
    const int src_lane = (lane & ~(G - 1)) | ((lane - 1) & (G - 1));
    auto claim = [&]() -> uint32_t {
      uint32_t w = 0;
      if (lane == 0) w = atomicAdd(&s_next, 1u);
      return __shfl_sync(FULL, w, 0);
    };
    uint32_t w_cur = claim();
    bool have = w_cur < task.wt_end;
    if (!have) {
      __syncthreads();
      continue;
    }
    Sw16WarpTask wt_cur = prm.warp_tasks[w_cur];
    Sw16Pair2 cur{};
    if (feeder) cur = load_pair2(prm, wt_cur.slot_begin, grp);
    uint32_t w_nxt = claim();
    bool have_nxt = w_nxt < task.wt_end;
    Sw16WarpTask wt_nxt = have_nxt ? prm.warp_tasks[w_nxt] : Sw16WarpTask{0, 0};
    Sw16Pair2 nxt{};
    if (have_nxt && feeder) nxt = load_pair2(prm, wt_nxt.slot_begin, grp);
    int u_col = 0, u_pass = 0, u_seq = 0, drain = 0;
    if (feeder) {
      s_pair[warp][grp][0][0] = cur.pA;
      s_pair[warp][grp][0][1] = cur.pB;
      s_best[warp][grp][0][0] = 0;
      s_best[warp][grp][0][1] = 0;
    }

    // per-lane wavefront state
    uint32_t Hp[R], E[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      Hp[k] = 0;
      E[k] = E0;
    }
    uint32_t best = 0, hup_prev = 0;
    // outgoing registers: a lane's outputs for the lane below (the feeder: lane 0's next inputs)
    uint32_t my_ctl = kCtlIdle, my_rA = SENTW, my_rB = SENTW;
    uint32_t my_h[C], my_f[C];
#pragma unroll
    for (int j = 0; j < C; ++j) {
      my_h[j] = 0;
      my_f[j] = F0;
    }
    if (feeder) {  // lane 0's first step: column 0, pass 0 of the first task
      my_ctl = 0u;
      my_rA = load_codes<C>(cur.tA, cur.lenA, 0);
      my_rB = load_codes<C>(cur.tB, cur.lenB, 0);
    }
    __syncwarp();

    for (;;) {
      // this step's inputs: from the lane above, lane 0 from the feeder
      const uint32_t ctl = __shfl_sync(FULL, my_ctl, src_lane);
      const uint32_t rA = __shfl_sync(FULL, my_rA, src_lane);
      const uint32_t rB = __shfl_sync(FULL, my_rB, src_lane);
      uint32_t h_in[C], f_in[C];
#pragma unroll
      for (int j = 0; j < C; ++j) {
        h_in[j] = __shfl_sync(FULL, my_h[j], src_lane);
        f_in[j] = __shfl_sync(FULL, my_f[j], src_lane);
      }
      my_ctl = ctl;
      my_rA = rA;
      my_rB = rB;
      const int col = static_cast<int>(ctl & 0xFFFFu);
      const int pass = static_cast<int>((ctl >> 16) & 0xFFu);
      // first column of a pass (or idle): left border H = 0, first-column E. The
      // groups of a warp move in step, so lane l of every group resets on the
      // same steps: the branch is skipped on the other steps of a pass.
      if (__any_sync(FULL, col == 0)) {
        if (col == 0) {
#pragma unroll
          for (int k = 0; k < R; ++k) {
            Hp[k] = 0;
            E[k] = E0;
          }
          hup_prev = 0;
        }
      }
      const int8_t* rows = prof_s + pass * (G * R) + gl * R;
#pragma unroll
      for (int j = 0; j < C; ++j) {
        const uint32_t resA = (rA >> (8 * j)) & 0xFFu;
        const uint32_t resB = (rB >> (8 * j)) & 0xFFu;
        uint32_t wa[Tile::kWords], wb[Tile::kWords];
        load_rows8<R>(rows + resA * m_pad, wa);
        load_rows8<R>(rows + resB * m_pad, wb);
        uint32_t hd = j == 0 ? hup_prev : h_in[j - 1];
        uint32_t F = f_in[j];
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
        my_h[j] = Hp[R - 1];
        my_f[j] = F;
      }
      hup_prev = h_in[C - 1];
      if (ctl & kCtlLast) {  // this lane's part of the task is done: fold its maximum into the task slot
        const int slot = static_cast<int>((ctl >> 24) & 7u);
        atomicMax(&s_best[warp][grp][slot][0], pk_lo(best));
        atomicMax(&s_best[warp][grp][slot][1], pk_hi(best));
        best = 0;
        if (feeder) {  // the group's last lane finishes the task last: report both scores
          const int32_t bA = s_best[warp][grp][slot][0], bB = s_best[warp][grp][slot][1];
          const uint32_t pA = s_pair[warp][grp][slot][0], pB = s_pair[warp][grp][slot][1];
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
      // the bottom row of a pass that is not the last goes to the scratch line
      if (feeder && !(ctl & kCtlIdle) && pass + 1 < P) store_bnd<C>(bnd + col, my_h, my_f);
      __syncwarp();

      // advance lane 0's stream position (uniform across the warp)
      if (have) {
        u_col += C;
        if (u_col == static_cast<int>(wt_cur.ncols)) {
          u_col = 0;
          if (++u_pass == P) {  // task done: the pre-claimed task becomes current, claim the one after
            u_pass = 0;
            ++u_seq;
            have = have_nxt;
            w_cur = w_nxt;
            wt_cur = wt_nxt;
            cur = nxt;
            if (have) {
              const int slot = u_seq & (kSlotRing - 1);
              if (feeder) {
                s_pair[warp][grp][slot][0] = cur.pA;
                s_pair[warp][grp][slot][1] = cur.pB;
                s_best[warp][grp][slot][0] = 0;
                s_best[warp][grp][slot][1] = 0;
              }
              w_nxt = claim();
              have_nxt = w_nxt < task.wt_end;
              if (have_nxt) {
                wt_nxt = prm.warp_tasks[w_nxt];
                if (feeder) nxt = load_pair2(prm, wt_nxt.slot_begin, grp);
              }
            }
          }
        }
      } else {
        ++drain;
      }
      if (!have && drain >= G) break;
      // the feeder's outgoing registers become lane 0's inputs for the next step
      if (feeder) {
        if (have) {
          const bool last = (u_pass == P - 1) && (u_col + C == static_cast<int>(wt_cur.ncols));
          my_ctl = static_cast<uint32_t>(u_col) | (static_cast<uint32_t>(u_pass) << 16) |
                   (static_cast<uint32_t>(u_seq & (kSlotRing - 1)) << 24) | (last ? kCtlLast : 0u);
          my_rA = load_codes<C>(cur.tA, cur.lenA, u_col);
          my_rB = load_codes<C>(cur.tB, cur.lenB, u_col);
          load_bnd<C>((u_pass > 0 ? bnd : prm.zline) + u_col, my_h, my_f);
        } else {
          my_ctl = kCtlIdle;
          my_rA = SENTW;
          my_rB = SENTW;
          load_bnd<C>(prm.zline, my_h, my_f);
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace st
