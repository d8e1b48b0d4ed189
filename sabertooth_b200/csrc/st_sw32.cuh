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
  // end-cell modes (sw32_end_kernel): the first optimum in column-major order
  // (src/simd.rs:375-381), -1 when the score is 0; in the reverse mode the
  // pair's query rows [0, rev_q] and target columns [0, rev_t] are scored
  // reversed (the start search of align_canonical, src/align.rs:848-866)
  int32_t* end_q;
  int32_t* end_t;
  const int32_t* rev_q;
  const int32_t* rev_t;
  // with band16 set, the entries [0, n_static) that sw16_band_kernel takes (banded pairs with int8 rows;
  // st_band16.cuh) were scored there and are skipped here
  uint32_t n_static = 0;
  uint32_t band16 = 0;
};

enum Sw32Mode { kSw32Score = 0, kSw32End = 1, kSw32RevEnd = 2 };

constexpr int kSw32G = 32;
constexpr int kSw32R = 8;
constexpr int kSw32Rows = kSw32G * kSw32R;  // rows per pass; profiles' int32 stride is a multiple of this

// (score, column, row) of a candidate optimum; a < b when a comes first: higher
// score, then smaller target column, then smaller query row
__device__ __forceinline__ bool end_before(int32_t s, int32_t c, int32_t r, int32_t bs, int32_t bc, int32_t br) {
  return s > bs || (s == bs && (c < bc || (c == bc && r < br)));
}

template <int MODE>
__device__ __forceinline__ void sw32_pair(const Sw32Params& prm, uint32_t p, int2* bnd) {
  constexpr int G = kSw32G, R = kSw32R;
  const int lane = threadIdx.x & 31;
  const uint32_t FULL = 0xFFFFFFFFu;
  const uint32_t q = prm.pair_query[p];
  const uint32_t tid = prm.pair_target[p];
  const int m_full = static_cast<int>(prm.prof.qlen[q]);
  const int n_full = static_cast<int>(prm.db.length[tid]);
  // the reverse mode scores the prefix [0, rev_q] x [0, rev_t], both reversed
  const int rq = MODE == kSw32RevEnd ? prm.rev_q[p] : 0;
  const int rt = MODE == kSw32RevEnd ? prm.rev_t[p] : 0;
  const int m = MODE == kSw32RevEnd ? (rq >= 0 ? min(rq + 1, m_full) : 0) : m_full;
  const int n = MODE == kSw32RevEnd ? (rt >= 0 ? min(rt + 1, n_full) : 0) : n_full;
  const int32_t center = MODE == kSw32Score ? prm.pair_center[p] : 0;
  const int32_t radius = MODE == kSw32Score ? prm.pair_radius[p] : -1;
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
      if (MODE != kSw32Score) {
        prm.end_q[p] = -1;
        prm.end_t[p] = -1;
      }
    }
    return;
  }
  const int cstart = static_cast<int>(c_lo);
  const int ncols = static_cast<int>(c_hi - c_lo);
  const int P = (m + G * R - 1) / (G * R);
  // Columns streamed per pass.  Lane 0 reads column c's boundary of pass p at
  // step p*W + c; lane G-1 wrote it at step (p-1)*W + c + G-1, which is earlier
  // only when W >= G.  A multi-pass query against fewer than G columns streams
  // idle columns [ncols, G) after the real ones: they carry the sentinel
  // residue, never count toward the maximum and never touch the boundary, and
  // the state they leave is reset when the next pass starts at column 0.
  const int W = P > 1 ? max(ncols, G) : ncols;
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
  int32_t bcol = 0x7FFFFFFF, brow = 0x7FFFFFFF;  // end modes: this lane's first optimum
  int c = -lane;
  int pass = 0;
  // target column j of the scored sequence (reversed in the reverse mode)
  auto tcol = [&](int j) -> uint32_t {
    const int jj = MODE == kSw32RevEnd ? rt - j : j;
    return min(static_cast<uint32_t>(__ldg(t + jj)), static_cast<uint32_t>(kSentinel));
  };
  // This lane's R profile scores of residue r at rows row0 .. row0 + R - 1.
  auto load_rows = [&](uint32_t r, int row0, int32_t (&S)[R]) {
    if constexpr (MODE == kSw32RevEnd) {
      // row i of the reversed query is row rq - i of the profile (rows past the prefix: any in-range row)
      const int32_t* rb = prof + static_cast<size_t>(r) * stride;
#pragma unroll
      for (int k = 0; k < R; ++k) S[k] = __ldg(rb + max(rq - (row0 + k), 0));
    } else {
      const int32_t* prow = prof + static_cast<size_t>(r) * stride + row0;
      const int4 a = __ldg(reinterpret_cast<const int4*>(prow));
      const int4 b = __ldg(reinterpret_cast<const int4*>(prow + 4));
      S[0] = a.x; S[1] = a.y; S[2] = a.z; S[3] = a.w;
      S[4] = b.x; S[5] = b.y; S[6] = b.z; S[7] = b.w;
    }
  };
  // Software pipeline: a step computes with the residue and profile scores loaded during the step before,
  // and loads the next step's.  A lane's next residue is the one its upper neighbour uses now (one extra
  // shuffle); lane 0 reads its target columns one more step ahead.  (c2, p2): lane 0's column and pass two
  // steps ahead.
  uint32_t res = kSentinel, q1 = kSentinel;
  int c2 = 2, p2 = 0;
  while (c2 >= W) {
    c2 -= W;
    ++p2;
  }
  if (lane == 0) {
    res = tcol(cstart);
    q1 = (1 < W) ? (1 < ncols ? tcol(cstart + 1) : kSentinel) : (1 < P ? tcol(cstart) : kSentinel);
  }
  int32_t S[R];
  load_rows(res, lane * R, S);
  const int steps = P * W + G - 1;

  for (int s = 0; s < steps; ++s) {
    int32_t hin = __shfl_up_sync(FULL, h_bot, 1);
    int32_t fin = __shfl_up_sync(FULL, f_out, 1);
    uint32_t rn = __shfl_up_sync(FULL, res, 1);  // the upper lane's residue now: this lane's next one
    if (lane == 0) {
      if (pass < P && pass > 0 && c < ncols) {
        const int2 bv = bnd[c];
        hin = bv.x;
        fin = bv.y;
      } else {
        hin = 0;
        fin = F0;
      }
      rn = q1;
      q1 = (p2 < P && c2 < ncols) ? tcol(cstart + c2) : kSentinel;
      if (++c2 == W) {
        c2 = 0;
        ++p2;
      }
    }
    // the next step's column and pass, and its profile scores
    int cn = c + 1, pn = pass;
    if (cn == W) {
      cn = 0;
      ++pn;
    }
    int32_t Sn[R];
    load_rows(rn, (pn < P ? pn : P - 1) * G * R + lane * R, Sn);
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
    const int col = cstart + c;  // target column (0-based) of this lane
    const bool live = (c >= 0) && (c < ncols) && (pass < P);
    // band rows of this column among the lane's R rows: row0 + k is in the band when
    // col - center - radius <= row0 + k <= col - center + radius, i.e. k_lo <= k <= k_hi (clamped to [-1, R])
    int k_lo = 0, k_hi = R - 1;
    if (banded) {
      const int64_t base = static_cast<int64_t>(col) - row0 - center;
      k_lo = static_cast<int>(i64max(-1, i64min(R, base - radius)));
      k_hi = static_cast<int>(i64max(-1, i64min(R, base + radius)));
    }
    int32_t hd = hup_prev;
    int32_t F = fin;
    int32_t lmax = 0;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int row = row0 + k;
      const bool inband = (k >= k_lo) && (k <= k_hi);
      const int32_t tt = max(wadd(hd, S[k]), E[k]);
      const int32_t Hc = max(max(tt, F), 0);
      const int32_t Ho = wsub(Hc, open);
      // out of the band: H = 0 and E = F = minus infinity (their successors then start from -open)
      const int32_t H = inband ? Hc : 0;
      const int32_t En = inband ? max(wsub(E[k], ext), Ho) : E0;
      const int32_t Fn = inband ? max(wsub(F, ext), Ho) : F0;
      if (row < m) {
        lmax = max(lmax, H);
        if constexpr (MODE != kSw32Score) {
          if (live && end_before(H, col, row, best, bcol, brow)) {
            best = H;
            bcol = col;
            brow = row;
          }
        }
      }
      E[k] = En;
      F = Fn;
      hd = Hp[k];
      Hp[k] = H;
    }
    if (MODE == kSw32Score && live) best = max(best, lmax);
    hup_prev = hin;
    h_bot = Hp[R - 1];
    f_out = F;
    if (lane == G - 1 && pass + 1 < P && c >= 0 && c < ncols) bnd[c] = make_int2(h_bot, f_out);
    c = cn;
    pass = pn;
    res = rn;
#pragma unroll
    for (int k = 0; k < R; ++k) S[k] = Sn[k];
    __syncwarp();
  }
  if constexpr (MODE == kSw32Score) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(FULL, best, o));
  } else {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const int32_t ob = __shfl_xor_sync(FULL, best, o);
      const int32_t oc = __shfl_xor_sync(FULL, bcol, o);
      const int32_t orow = __shfl_xor_sync(FULL, brow, o);
      if (end_before(ob, oc, orow, best, bcol, brow)) {
        best = ob;
        bcol = oc;
        brow = orow;
      }
    }
  }
  if (lane == 0) {
    prm.scores[p] = best;
    if (prm.kernels) prm.kernels[p] = 2u;
    if (MODE != kSw32Score) {
      prm.end_q[p] = best > 0 ? brow : -1;
      prm.end_t[p] = best > 0 ? bcol : -1;
    }
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
    const uint32_t p = prm.list[w];
    // banded pairs with int8 rows of the static list: scored by the packed band kernel
    if (prm.band16 && w < prm.n_static && prm.pair_radius[p] >= 0 && prm.prof.fits8[prm.pair_query[p]] != 0)
      continue;
    sw32_pair<kSw32Score>(prm, p, bnd);
  }
}

// Score and end cell of every listed pair (MODE kSw32End), or of the reversed
// prefixes ending at (rev_q, rev_t) (MODE kSw32RevEnd). Unbanded pairs only.
template <int WARPS, int MODE>
__global__ void __launch_bounds__(WARPS * 32) sw32_end_kernel(const Sw32Params prm) {
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int2* bnd = prm.scratch + static_cast<size_t>(blockIdx.x * WARPS + warp) * prm.scratch_stride;
  const uint32_t count = *prm.list_count;
  for (;;) {
    uint32_t w = 0;
    if (lane == 0) w = atomicAdd(prm.work_counter, 1u);
    w = __shfl_sync(0xFFFFFFFFu, w, 0);
    if (w >= count) break;
    sw32_pair<MODE>(prm, prm.list[w], bnd);
  }
}

}  // namespace st
