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
          const uint4 v = *reinterpret_cast<const uint4*>(tp + pa);
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

}  // namespace st
