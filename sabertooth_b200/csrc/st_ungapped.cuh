// Ungapped diagonal scoring (the reference's ungapped::score_batch /
// kadane_score, src/ungapped.rs:53-62 and 285-386).
//
// One thread scores one diagonal: Kadane's running maximum
//   cur = max(cur, 0) + s(q, t[q + d]),  best = max(best, cur),  best0 = 0
// over query positions [lo, hi), exactly as kadane_score, in int32 (the GPU
// needs no u8 headroom and no rescore).  Target residues are read as aligned
// 16-byte vectors from the padded database arena; cells of a vector that lie
// outside [lo, hi) score 0, which cannot change the result (the reference's
// SENTINEL argument, src/ungapped.rs:28-33).
//
// A CTA takes a chunk of jobs; jobs are expected sorted by query (the order
// the prefilter produces), and each run of one query inside the chunk stages
// that query's int8 profile in shared memory (residue-major, 16 guard bytes on
// each side of every row so out-of-window positions stay inside the array).
#pragma once
#include "st_common.cuh"

namespace st {

struct UngappedJob {  // explicit window (the drop-in lanes)
  uint32_t query;
  uint32_t target;
  int32_t diag;
  uint32_t lo;
  uint32_t hi;
};

struct HitRec {  // a prefilter seed hit: the window is the whole diagonal
  uint32_t query;
  uint32_t target;
  int32_t diag;
};

struct UngappedParams {
  DeviceDb db;
  DeviceProfiles prof;
  const void* jobs;  // UngappedJob[] or HitRec[]
  uint64_t n;
  int32_t* out;
  uint32_t max_m_pad;  // row stride of the staged profile (>= every query length + 32)
};

constexpr int kUngChunk = 1024;  // jobs per CTA chunk

template <bool HITS>
__device__ __forceinline__ void ung_job(const UngappedParams& prm, uint64_t k, uint32_t& q, uint32_t& t,
                                        int32_t& d, int64_t& lo, int64_t& hi) {
  if constexpr (HITS) {
    const HitRec h = reinterpret_cast<const HitRec*>(prm.jobs)[k];
    q = h.query;
    t = h.target;
    d = h.diag;
    const int64_t m = prm.prof.qlen[q];
    const int64_t n = prm.db.length[t];
    // diag_range, src/ungapped.rs:38-46
    lo = i64max(-static_cast<int64_t>(d), 0);
    hi = i64min(m, n - d);
    if (hi <= lo) lo = hi = 0;
  } else {
    const UngappedJob j = reinterpret_cast<const UngappedJob*>(prm.jobs)[k];
    q = j.query;
    t = j.target;
    d = j.diag;
    lo = j.lo;
    hi = j.hi;
  }
}

template <bool HITS>
__device__ __forceinline__ uint32_t ung_query(const UngappedParams& prm, uint64_t k) {
  if constexpr (HITS)
    return reinterpret_cast<const HitRec*>(prm.jobs)[k].query;
  else
    return reinterpret_cast<const UngappedJob*>(prm.jobs)[k].query;
}

template <bool HITS>
__global__ void __launch_bounds__(256) ungapped_kernel(const UngappedParams prm) {
  extern __shared__ __align__(16) int8_t smem[];
  __shared__ uint32_t s_run_end;
  const uint32_t stride = prm.max_m_pad;
  int8_t* base = smem + 16;  // 16 guard bytes before row 0
  const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * kUngChunk;
  if (c0 >= prm.n) return;
  const uint64_t c1 = u64min(prm.n, c0 + kUngChunk);
  uint64_t a = c0;
  while (a < c1) {
    const uint32_t q = ung_query<HITS>(prm, a);
    // end of this query's run inside the chunk (warp 0 scans 32 jobs at a time)
    if (threadIdx.x < 32) {
      uint64_t e = a;
      for (;;) {
        const uint64_t k = e + threadIdx.x;
        const bool same = (k < c1) && (ung_query<HITS>(prm, k) == q);
        const uint32_t ball = __ballot_sync(0xFFFFFFFFu, same);
        if (ball != 0xFFFFFFFFu) {
          e += __ffs(~ball) - 1;
          break;
        }
        e += 32;
      }
      if (threadIdx.x == 0) s_run_end = static_cast<uint32_t>(e - c0);
    }
    // stage the profile of q: rows 0..21, m entries each, zero elsewhere
    const uint32_t m = prm.prof.qlen[q];
    const uint32_t pstride = prm.prof.stride8[q];
    const int8_t* src = prm.prof.p8[q];
    for (uint32_t idx = threadIdx.x; idx < kProfRows * (stride / 16); idx += blockDim.x) {
      const uint32_t r = idx / (stride / 16);
      const uint32_t i = (idx - r * (stride / 16)) * 16;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (i < pstride) v = *reinterpret_cast<const uint4*>(src + static_cast<size_t>(r) * pstride + i);
      *reinterpret_cast<uint4*>(base + static_cast<size_t>(r) * stride + i) = v;
    }
    if (threadIdx.x < 16) {  // guard bytes before row 0
      smem[threadIdx.x] = 0;
    }
    __syncthreads();
    const uint64_t b = c0 + s_run_end;
    // rows outside int8 (rare: composition-corrected or custom rows) read the int32 profile from global memory
    const bool narrow = prm.prof.fits8[q] != 0;
    const int32_t* p32 = prm.prof.p32[q];
    const int32_t s32 = static_cast<int32_t>(prm.prof.stride32[q]);
    const int32_t last_row = static_cast<int32_t>(m) - 1;
    for (uint64_t k = a + threadIdx.x; k < b; k += blockDim.x) {
      uint32_t qq, tt;
      int32_t d;
      int64_t lo, hi;
      ung_job<HITS>(prm, k, qq, tt, d, lo, hi);
      int32_t best = 0, cur = 0;
      if (HITS && hi > lo && narrow) {
        // Whole-diagonal windows (hits) on int8 profiles: every cell of a vector outside [lo, hi) scores
        // 0 on its own: query rows before 0 or from m read the zero guard bytes and padding of the staged
        // rows, target positions from n hold the sentinel code, whose row is zero. Zero cells at either
        // end of the window cannot change Kadane's maximum, so whole vectors are scored without a test.
        const uint8_t* tp = prm.db.arena + prm.db.offset[tt];
        const int32_t p0 = static_cast<int32_t>(lo) + d, p1 = static_cast<int32_t>(hi) + d;
        for (int32_t pa = p0 & ~15; pa < p1; pa += 16) {
          const uint4 v = *reinterpret_cast<const uint4*>(tp + pa);
          const uint32_t w[4] = {v.x, v.y, v.z, v.w};
          const int8_t* rowbase = base + (pa - d);
#pragma unroll
          for (int bb = 0; bb < 16; ++bb) {
            const uint32_t r = (w[bb >> 2] >> ((bb & 3) * 8)) & 0xFFu;
            const int32_t sc = rowbase[static_cast<int32_t>(r * stride) + bb];
            cur = wadd(max(cur, 0), sc);
            best = max(best, cur);
          }
        }
      } else if (hi > lo) {
        const uint8_t* tp = prm.db.arena + prm.db.offset[tt];
        // target positions [p0, p1); sequences are shorter than 2^31
        const int32_t p0 = static_cast<int32_t>(lo) + d, p1 = static_cast<int32_t>(hi) + d;
        int32_t pa = p0 & ~15;
        for (; pa < p1; pa += 16) {
          const uint4 v = *reinterpret_cast<const uint4*>(tp + pa);
          const uint32_t w[4] = {v.x, v.y, v.z, v.w};
          const int32_t qa = pa - d;  // query row of the vector's first byte
          const int8_t* rowbase = base + qa;
#pragma unroll
          for (int bb = 0; bb < 16; ++bb) {
            const uint32_t r = (w[bb >> 2] >> ((bb & 3) * 8)) & 0xFFu;
            const int32_t p = pa + bb;
            const bool in = (p >= p0) && (p < p1);
            int32_t sc;
            if (narrow) {
              sc = rowbase[static_cast<int32_t>(r * stride) + bb];
            } else {
              const int32_t row = min(max(qa + bb, 0), last_row);
              sc = __ldg(p32 + static_cast<int32_t>(r) * s32 + row);
            }
            const int32_t s = in ? sc : 0;
            cur = wadd(max(cur, 0), s);
            best = max(best, cur);
          }
        }
      }
      prm.out[k] = best;
    }
    __syncthreads();
    a = b;
  }
}

// Hits (whole-diagonal windows, diag_range) with one hit per lane: per run of
// one query inside the CTA's chunk the profile is staged as above, then every
// lane keeps a hit in flight, one 16-byte target vector per step, and takes the
// run's next hit from a shared counter as soon as its own is done, so lanes
// stay busy whatever the diagonal lengths.  On int8 profiles no cell needs a
// test (the argument of the whole-diagonal path of ungapped_kernel); rows
// outside int8 read the int32 profile with an explicit window test.
__global__ void __launch_bounds__(256) ungapped_hits_refill_kernel(const UngappedParams prm) {
  extern __shared__ __align__(16) int8_t smem[];
  __shared__ unsigned long long s_run_end;
  __shared__ uint32_t s_next;
  const HitRec* hits = reinterpret_cast<const HitRec*>(prm.jobs);
  const uint32_t stride = prm.max_m_pad;
  int8_t* base = smem + 16;
  const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * kUngChunk;
  if (c0 >= prm.n) return;
  const uint64_t c1 = u64min(prm.n, c0 + kUngChunk);
  uint64_t a = c0;
  while (a < c1) {
    const uint32_t q = hits[a].query;
    if (threadIdx.x < 32) {
      uint64_t e = a;
      for (;;) {
        const uint64_t k = e + threadIdx.x;
        const bool same = (k < c1) && (hits[k].query == q);
        const uint32_t ball = __ballot_sync(0xFFFFFFFFu, same);
        if (ball != 0xFFFFFFFFu) {
          e += __ffs(~ball) - 1;
          break;
        }
        e += 32;
      }
      if (threadIdx.x == 0) {
        s_run_end = e;
        s_next = blockDim.x;
      }
    }
    const uint32_t m = prm.prof.qlen[q];
    const uint32_t pstride = prm.prof.stride8[q];
    const int8_t* src = prm.prof.p8[q];
    for (uint32_t idx = threadIdx.x; idx < kProfRows * (stride / 16); idx += blockDim.x) {
      const uint32_t r = idx / (stride / 16);
      const uint32_t i = (idx - r * (stride / 16)) * 16;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (i < pstride) v = *reinterpret_cast<const uint4*>(src + static_cast<size_t>(r) * pstride + i);
      *reinterpret_cast<uint4*>(base + static_cast<size_t>(r) * stride + i) = v;
    }
    if (threadIdx.x < 16) smem[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t b = s_run_end;
    const uint32_t nb = static_cast<uint32_t>(b - a);  // hits of the run, indexed from a
    const HitRec* run = hits + a;
    const bool narrow = prm.prof.fits8[q] != 0;
    const int32_t* p32 = prm.prof.p32[q];
    const int32_t s32 = static_cast<int32_t>(prm.prof.stride32[q]);
    const int32_t last_row = static_cast<int32_t>(m) - 1;
    uint32_t k = threadIdx.x;
    const uint8_t* tp = nullptr;
    int32_t d = 0, p0 = 0, p1 = 0, pa = 0, cur = 0, best = 0;
    uint4 vnext = make_uint4(0, 0, 0, 0);  // the lane's next target vector, requested a step ahead
    bool live = false;
    auto take = [&](uint32_t j) {
      k = j;
      live = j < nb;
      if (live) {
        const HitRec h = run[j];
        const int64_t n = prm.db.length[h.target];
        d = h.diag;
        // diag_range, src/ungapped.rs:38-46
        const int64_t lo = i64max(-static_cast<int64_t>(d), 0), hi = i64min(m, n - d);
        tp = prm.db.arena + prm.db.offset[h.target];
        if (hi > lo) {
          p0 = static_cast<int32_t>(lo) + d;
          p1 = static_cast<int32_t>(hi) + d;
          pa = p0 & ~15;
          vnext = *reinterpret_cast<const uint4*>(tp + pa);
        } else {
          p0 = p1 = pa = 0;  // empty: done at once
        }
        cur = 0;
        best = 0;
      }
    };
    take(k);
    while (__any_sync(0xFFFFFFFFu, live)) {
      if (live) {
        if (pa < p1) {
          // the vector loaded one step ago; the next one is requested before this one is scored
          const uint4 v = vnext;
          if (pa + 16 < p1) vnext = *reinterpret_cast<const uint4*>(tp + pa + 16);
          const uint32_t w[4] = {v.x, v.y, v.z, v.w};
          const int32_t qa = pa - d;
          if (narrow) {
            // u = max(cur, 0) carried instead of cur: u' = max(u + s, 0) is one DPX op, and
            // max(best, cur) = max(best, u) since best >= 0; int8 scores over at most 2^20 rows
            // cannot overflow, so the unwrapped add equals the reference's wrapping one
            const int8_t* rowbase = base + qa;
#pragma unroll
            for (int bb = 0; bb < 16; bb += 2) {
              const uint32_t r0 = (w[bb >> 2] >> ((bb & 3) * 8)) & 0xFFu;
              const uint32_t r1 = (w[bb >> 2] >> (((bb + 1) & 3) * 8)) & 0xFFu;
              const int32_t u0 =
                  __viaddmax_s32_relu(cur, static_cast<int32_t>(rowbase[static_cast<int32_t>(r0 * stride) + bb]), 0);
              cur = __viaddmax_s32_relu(u0, static_cast<int32_t>(rowbase[static_cast<int32_t>(r1 * stride) + bb + 1]),
                                        0);
              best = __vimax3_s32(best, u0, cur);
            }
          } else {
#pragma unroll
            for (int bb = 0; bb < 16; ++bb) {
              const uint32_t r = (w[bb >> 2] >> ((bb & 3) * 8)) & 0xFFu;
              const int32_t p = pa + bb;
              const int32_t row = min(max(qa + bb, 0), last_row);
              const int32_t sc = (p >= p0 && p < p1) ? __ldg(p32 + static_cast<int32_t>(r) * s32 + row) : 0;
              cur = wadd(max(cur, 0), sc);
              best = max(best, cur);
            }
          }
          pa += 16;
        }
        if (pa >= p1) {
          prm.out[a + k] = best;
          take(atomicAdd(&s_next, 1u));
        }
      }
    }
    __syncthreads();
    a = b;
  }
}


// Hits with the work of a query run split evenly over the CTA's lanes.
//
// Per run of one query inside the CTA's chunk: the profile is staged as
// above; every hit of the run is decoded once (diag_range, the first aligned
// target vector, the number of 16-byte vectors) into shared memory, and an
// exclusive scan of the vector counts lays the run's vectors end to end.  Lane
// t then scores vectors [t*S, (t+1)*S) of that stream, S = ceil(V / lanes), so
// every lane does the same work whatever the diagonal lengths; a diagonal may
// be split over consecutive lanes.
//
// Splitting is exact.  With u = max(cur, 0) carried (u' = max(u + s, 0)) and
// any u_in >= 0, the states after k cells are u_k = max(u_in + P_k, z_k), where
// P_k is the k-th prefix sum of the cell scores and z_k the state of the same
// cells scored from u = 0; the best over the piece is max(u_in + C, D) with
// C = max_k P_k and D = max_k z_k.  A lane that starts inside a diagonal scores
// its piece from 0 (giving z, D) and from a large H (u never reaches 0 from
// there, so that run carries H + P_k and its maximum H + C), and stores
// (A = P_last, B = z_last, C, D).  After one barrier the lane that started the
// diagonal folds the summaries of the lanes after it in order: best = max(best,
// u + C, D), u = max(u + A, B), which is Kadane's result over the whole
// diagonal (src/ungapped.rs:53-62).  Rows outside int8 take the plain loop.
constexpr int kUngSplitLanes = 256;
constexpr int32_t kUngH = 1 << 24;  // > 127 * rows of any staged profile: H + P_k stays positive

__global__ void __launch_bounds__(kUngSplitLanes) ungapped_hits_split_kernel(const UngappedParams prm) {
  extern __shared__ __align__(16) int8_t smem[];
  __shared__ unsigned long long s_run_end;
  __shared__ unsigned long long s_vec0[kUngChunk];  // arena offset of the hit's first (aligned) vector
  __shared__ int32_t s_qa0[kUngChunk];               // query row of that vector's first byte
  __shared__ uint32_t s_vstart[kUngChunk + 1];       // exclusive scan of the vector counts
  __shared__ int4 s_sum[kUngSplitLanes];             // (A, B, C, D) of a lane's leading piece
  __shared__ uint32_t s_warp[kUngSplitLanes / 32];
  const HitRec* hits = reinterpret_cast<const HitRec*>(prm.jobs);
  const uint32_t stride = prm.max_m_pad;
  int8_t* base = smem + 16;
  const int t = threadIdx.x;
  const int lane = t & 31, warp = t >> 5;
  const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * kUngChunk;
  if (c0 >= prm.n) return;
  const uint64_t c1 = u64min(prm.n, c0 + kUngChunk);
  uint64_t a = c0;
  while (a < c1) {
    const uint32_t q = hits[a].query;
    if (t < 32) {
      uint64_t e = a;
      for (;;) {
        const uint64_t k = e + lane;
        const bool same = (k < c1) && (hits[k].query == q);
        const uint32_t ball = __ballot_sync(0xFFFFFFFFu, same);
        if (ball != 0xFFFFFFFFu) {
          e += __ffs(~ball) - 1;
          break;
        }
        e += 32;
      }
      if (t == 0) s_run_end = e;
    }
    const uint32_t m = prm.prof.qlen[q];
    const uint32_t pstride = prm.prof.stride8[q];
    const int8_t* src = prm.prof.p8[q];
    for (uint32_t idx = t; idx < kProfRows * (stride / 16); idx += blockDim.x) {
      const uint32_t r = idx / (stride / 16);
      const uint32_t i = (idx - r * (stride / 16)) * 16;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (i < pstride) v = *reinterpret_cast<const uint4*>(src + static_cast<size_t>(r) * pstride + i);
      *reinterpret_cast<uint4*>(base + static_cast<size_t>(r) * stride + i) = v;
    }
    if (t < 16) smem[t] = 0;
    __syncthreads();
    const uint64_t b = s_run_end;
    const uint32_t nb = static_cast<uint32_t>(b - a);
    const HitRec* run = hits + a;
    int32_t* out = prm.out + a;
    if (prm.prof.fits8[q] == 0) {
      // rows outside int8: the int32 profile, every cell tested against the window
      const int32_t* p32 = prm.prof.p32[q];
      const int32_t s32 = static_cast<int32_t>(prm.prof.stride32[q]);
      for (uint32_t j = t; j < nb; j += blockDim.x) {
        const HitRec h = run[j];
        const int64_t n = prm.db.length[h.target];
        const int64_t lo = i64max(-static_cast<int64_t>(h.diag), 0), hi = i64min(m, n - h.diag);
        int32_t cur = 0, best = 0;
        const uint8_t* tp = prm.db.arena + prm.db.offset[h.target];
        for (int64_t i = lo; i < hi; ++i) {
          const uint32_t r = tp[i + h.diag];
          cur = wadd(max(cur, 0), __ldg(p32 + static_cast<int32_t>(r) * s32 + static_cast<int32_t>(i)));
          best = max(best, cur);
        }
        out[j] = best;
      }
      __syncthreads();
      a = b;
      continue;
    }
    // decode: four consecutive hits per lane, so the scan below is a lane-local sum plus a block scan
    uint32_t cnt[4];
    uint32_t tot = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint32_t j = 4 * t + i;
      cnt[i] = 0;
      if (j < nb) {
        const HitRec h = run[j];
        const int64_t n = prm.db.length[h.target];
        // diag_range, src/ungapped.rs:38-46
        const int64_t lo = i64max(-static_cast<int64_t>(h.diag), 0), hi = i64min(m, n - h.diag);
        if (hi > lo) {
          const int32_t p0 = static_cast<int32_t>(lo) + h.diag, p1 = static_cast<int32_t>(hi) + h.diag;
          const int32_t pa = p0 & ~15;
          s_vec0[j] = prm.db.offset[h.target] + static_cast<uint64_t>(pa);
          s_qa0[j] = pa - h.diag;
          cnt[i] = static_cast<uint32_t>((p1 - pa + 15) >> 4);
        } else {
          out[j] = 0;  // an empty diagonal scores 0
        }
      }
      tot += cnt[i];
    }
    // block-wide exclusive scan of the lanes' totals
    uint32_t incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t wbase = 0, V = 0;
#pragma unroll
    for (int w = 0; w < kUngSplitLanes / 32; ++w) {
      const uint32_t x = s_warp[w];
      wbase += w < warp ? x : 0;
      V += x;
    }
    uint32_t run_start = wbase + incl - tot;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint32_t j = 4 * t + i;
      if (j < nb) s_vstart[j] = run_start;
      run_start += cnt[i];
    }
    if (t == 0) s_vstart[nb] = V;
    __syncthreads();
    const uint32_t S = (V + kUngSplitLanes - 1) / kUngSplitLanes;
    const uint32_t v0 = static_cast<uint32_t>(t) * S;
    const uint32_t v1 = min(v0 + S, V);
    bool tail = false;  // this lane started a diagonal that continues past its range
    uint32_t tail_h = 0;
    int32_t tail_u = 0, tail_b = 0;
    if (v0 < v1) {
      // the hit holding vector v0: the last one whose first vector is at or before v0 (hits with no vectors
      // share their successor's start and are passed over)
      uint32_t lo_i = 0, hi_i = nb;  // s_vstart[lo_i] <= v0 < s_vstart[hi_i]
      while (hi_i - lo_i > 1) {
        const uint32_t mid = (lo_i + hi_i) >> 1;
        if (s_vstart[mid] <= v0) lo_i = mid; else hi_i = mid;
      }
      uint32_t h = lo_i;
      while (s_vstart[h + 1] <= v0) ++h;
      uint32_t hend = s_vstart[h + 1];
      uint32_t w0 = v0 - s_vstart[h];
      bool head = w0 > 0;  // a piece of a diagonal that an earlier lane started
      const uint8_t* tp = prm.db.arena + s_vec0[h] + 16u * w0;
      const int8_t* rowbase = base + s_qa0[h] + 16 * static_cast<int32_t>(w0);
      int32_t u = 0, best = 0, uh = kUngH, bh = 0;
      for (uint32_t v = v0; v < v1;) {
        const uint4 vec = *reinterpret_cast<const uint4*>(tp);
        const uint32_t w[4] = {vec.x, vec.y, vec.z, vec.w};
        // every cell of a whole vector is scored: cells outside the window score 0 (guard bytes and padding
        // of the staged rows, sentinel residues past the target), which cannot change Kadane's result
#pragma unroll
        for (int bb = 0; bb < 16; bb += 2) {
          const uint32_t r0 = (w[bb >> 2] >> ((bb & 3) * 8)) & 0xFFu;
          const uint32_t r1 = (w[bb >> 2] >> (((bb + 1) & 3) * 8)) & 0xFFu;
          const int32_t s0 = rowbase[static_cast<int32_t>(r0 * stride) + bb];
          const int32_t s1 = rowbase[static_cast<int32_t>(r1 * stride) + bb + 1];
          const int32_t u0 = __viaddmax_s32_relu(u, s0, 0);
          u = __viaddmax_s32_relu(u0, s1, 0);
          best = __vimax3_s32(best, u0, u);
          const int32_t h0 = uh + s0;
          uh = h0 + s1;
          bh = __vimax3_s32(bh, h0, uh);
        }
        ++v;
        tp += 16;
        rowbase += 16;
        if (v == hend) {
          if (head) {
            s_sum[t] = make_int4(uh - kUngH, u, bh - kUngH, best);
            head = false;
          } else {
            out[h] = best;
          }
          ++h;
          while (h < nb && s_vstart[h + 1] == s_vstart[h]) ++h;
          if (v < v1) {
            hend = s_vstart[h + 1];
            tp = prm.db.arena + s_vec0[h];
            rowbase = base + s_qa0[h];
            u = 0;
            best = 0;
            uh = kUngH;
            bh = 0;
          }
        }
      }
      if (v1 < hend) {  // the range ended inside diagonal h
        if (head) {
          s_sum[t] = make_int4(uh - kUngH, u, bh - kUngH, best);
        } else {
          tail = true;
          tail_h = h;
          tail_u = u;
          tail_b = best;
        }
      }
    }
    __syncthreads();
    if (tail) {
      const uint32_t t_last = (s_vstart[tail_h + 1] - 1) / S;
      int32_t u = tail_u, best = tail_b;
      for (uint32_t tt = t + 1; tt <= t_last; ++tt) {
        const int4 sm = s_sum[tt];
        best = max(best, max(u + sm.z, sm.w));
        u = max(u + sm.x, sm.y);
      }
      out[tail_h] = best;
    }
    __syncthreads();
    a = b;
  }
}

}  // namespace st
