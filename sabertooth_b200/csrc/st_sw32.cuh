// Exact 32-bit Smith-Waterman-Gotoh score kernel: the rescore path for pairs
// whose 16-bit cells reached the headroom limit, for score rows outside int8,
// for gap costs outside the 16-bit kernel's range, and for the heuristic band
// of local_align_in_band.  It computes the reference's scalar recurrence
// (src/simd.rs:347-390) cell for cell in wrapping int32 with the same
// "minus infinity" i32::MIN/4, and the band rule of local_full_tb
// (src/align.rs:439-447): a cell with |j - i - center| > radius (1-based) has
// H = 0 and resets E and F to minus infinity.
//
// One warp scores one pair; lane l owns rows [pass*256 + 8l, +8) of the query
// and the target streams through the warp as a wavefront (as in the 16-bit
// kernel, one target per register instead of two).  Only real cells (row < m,
// column < n, inside the band) update the maximum, so the result is exact for
// any gap costs.  With a band, only columns that hold band cells are streamed:
// every cell left of them is outside the band and leaves the state that the
// first streamed column starts from.
#pragma once
#include "st_common.cuh"

namespace st {

struct Sw32Params {
  DeviceDb db;
  DeviceProfiles prof;
  const uint32_t* list;        // pair indices to score
  const uint32_t* list_count;  // device count of list (read at run time)
  const uint32_t* pair_query;
  const uint32_t* pair_target;
  const int32_t* pair_center;
  const int32_t* pair_radius;  // < 0: no band
  int32_t* scores;
  uint32_t* kernels;
  uint32_t* work_counter;
  int2* scratch;  // pass boundary rows, scratch_stride per warp
  uint32_t scratch_stride;
  int32_t open, ext;
};

constexpr int kSw32G = 32;
constexpr int kSw32R = 8;
constexpr int kSw32Rows = kSw32G * kSw32R;  // rows per pass; profiles' int32 stride is a multiple of this

__device__ __forceinline__ void sw32_pair(const Sw32Params& prm, uint32_t p, int2* bnd) {
  constexpr int G = kSw32G, R = kSw32R;
  const int lane = threadIdx.x & 31;
  const uint32_t FULL = 0xFFFFFFFFu;
  const uint32_t q = prm.pair_query[p];
  const uint32_t tid = prm.pair_target[p];
  const int m = static_cast<int>(prm.prof.qlen[q]);
  const int n = static_cast<int>(prm.db.length[tid]);
  const int32_t center = prm.pair_center[p];
  const int32_t radius = prm.pair_radius[p];
  const bool banded = radius >= 0;
  // columns that can hold band cells: row + center - radius .. row + center + radius
  int64_t c_lo = 0, c_hi = n;  // [c_lo, c_hi)
  if (banded) {
    c_lo = i64max(0, static_cast<int64_t>(center) - radius);
    c_hi = i64min(n, static_cast<int64_t>(m) - 1 + center + radius + 1);
  }
  if (m == 0 || n == 0 || c_hi <= c_lo) {
    if (lane == 0) {
      prm.scores[p] = 0;
      if (prm.kernels) prm.kernels[p] = 2u;
    }
    return;
  }
  const int cstart = static_cast<int>(c_lo);
  const int ncols = static_cast<int>(c_hi - c_lo);
  const int P = (m + G * R - 1) / (G * R);
  const uint8_t* t = prm.db.arena + prm.db.offset[tid];
  const int32_t* prof = prm.prof.p32[q];
  const uint32_t stride = prm.prof.stride32[q];
  const int32_t open = prm.open, ext = prm.ext;
  const int32_t E0 = max(wsub(0, open), wsub(kNeg32, ext));  // E of a first column / after a band reset
  const int32_t F0 = E0;                                     // F of a first row / after a band reset

  int32_t Hp[R], E[R];
#pragma unroll
  for (int k = 0; k < R; ++k) {
    Hp[k] = 0;
    E[k] = E0;
  }
  int32_t best = 0, hup_prev = 0, h_bot = 0, f_out = F0;
  uint32_t res = kSentinel;
  int c = -lane;
  int pass = 0;
  uint32_t nxt = kSentinel;
  if (lane == 0) nxt = min(static_cast<uint32_t>(__ldg(t + cstart)), static_cast<uint32_t>(kSentinel));
  const int steps = P * ncols + G - 1;

  for (int s = 0; s < steps; ++s) {
    int32_t hin = __shfl_up_sync(FULL, h_bot, 1);
    int32_t fin = __shfl_up_sync(FULL, f_out, 1);
    uint32_t rin = __shfl_up_sync(FULL, res, 1);
    if (lane == 0) {
      if (pass < P) {
        rin = nxt;
        int cn = c + 1;
        bool last = (cn == ncols);
        if (last) cn = 0;
        nxt = (last && pass + 1 >= P)
                  ? kSentinel
                  : min(static_cast<uint32_t>(__ldg(t + cstart + cn)), static_cast<uint32_t>(kSentinel));
        if (pass > 0) {
          int2 bv = bnd[c];
          hin = bv.x;
          fin = bv.y;
        } else {
          hin = 0;
          fin = F0;
        }
      } else {
        rin = kSentinel;
        hin = 0;
        fin = F0;
      }
    }
    res = rin;
    if (c == 0) {
#pragma unroll
      for (int k = 0; k < R; ++k) {
        Hp[k] = 0;
        E[k] = E0;
      }
      hup_prev = 0;
    }
    const int pp = pass < P ? pass : P - 1;
    const int row0 = pp * G * R + lane * R;
    const int32_t* prow = prof + static_cast<size_t>(res) * stride + row0;
    int32_t S[R];
    {
      const int4 a = __ldg(reinterpret_cast<const int4*>(prow));
      const int4 b = __ldg(reinterpret_cast<const int4*>(prow + 4));
      S[0] = a.x; S[1] = a.y; S[2] = a.z; S[3] = a.w;
      S[4] = b.x; S[5] = b.y; S[6] = b.z; S[7] = b.w;
    }
    const int col = cstart + c;  // target column (0-based) of this lane
    const bool live = (c >= 0) && (pass < P);
    int32_t hd = hup_prev;
    int32_t F = fin;
    int32_t lmax = 0;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int row = row0 + k;
      int32_t H, En, Fn;
      bool inband = true;
      if (banded) {
        const int64_t off = static_cast<int64_t>(col) - row - center;
        inband = (off >= -radius) && (off <= radius);
      }
      if (inband) {
        const int32_t tt = max(wadd(hd, S[k]), E[k]);
        H = max(max(tt, F), 0);
        const int32_t Ho = wsub(H, open);
        En = max(wsub(E[k], ext), Ho);
        Fn = max(wsub(F, ext), Ho);
        if (row < m) lmax = max(lmax, H);
      } else {
        H = 0;
        En = E0;
        Fn = F0;
      }
      E[k] = En;
      F = Fn;
      hd = Hp[k];
      Hp[k] = H;
    }
    if (live) best = max(best, lmax);
    hup_prev = hin;
    h_bot = Hp[R - 1];
    f_out = F;
    if (lane == G - 1 && pass + 1 < P && c >= 0) bnd[c] = make_int2(h_bot, f_out);
    if (++c == ncols) {
      c = 0;
      ++pass;
    }
    __syncwarp();
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(FULL, best, o));
  if (lane == 0) {
    prm.scores[p] = best;
    if (prm.kernels) prm.kernels[p] = 2u;
  }
}

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) sw32_kernel(const Sw32Params prm) {
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int2* bnd = prm.scratch + static_cast<size_t>(blockIdx.x * WARPS + warp) * prm.scratch_stride;
  const uint32_t count = *prm.list_count;
  for (;;) {
    uint32_t w = 0;
    if (lane == 0) w = atomicAdd(prm.work_counter, 1u);
    w = __shfl_sync(0xFFFFFFFFu, w, 0);
    if (w >= count) break;
    sw32_pair(prm, prm.list[w], bnd);
  }
}

}  // namespace st
