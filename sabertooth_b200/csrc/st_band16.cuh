// Banded pairs in packed 16-bit cells: two pairs per warp, one per half.
//
// The heuristic band of local_align_in_band (src/align.rs:439-447: a cell with
// |j - i - center| > radius, 1-based, has H = 0 and resets E and F to minus
// infinity) leaves a band of 2*radius + 1 cells per row; pairs carrying it
// have their own query each in the long/overflow mix, so the 16-bit tile
// classes (which share one query's staged profile among many targets) do not
// fit them.  Here one warp scores two banded pairs at once, one per 16-bit
// half of every register, with the geometry of the exact 32-bit kernel: lane l
// owns query rows [pass*256 + 8l, +8), the columns of both pairs' band windows
// stream through the warp as a wavefront, and a query of more than 256 rows
// is scored in passes whose bottom row goes through the warp's scratch line.
// The recurrence is the packed one of the tile classes (six DPX operations and
// a prmt per cell pair); a per-cell band mask, built per lane and step from
// the band rows of the lane's eight rows, sets out-of-band cells to H = 0 and
// their successors' E and F to -open, as the 32-bit kernel does.
//
// Exactness.  The int8 scores come from the profile's int8 layout (pairs whose
// rows do not fit int8 stay with the 32-bit kernel), the gap costs are within
// the 16-bit range (checked on the host), and a half whose best H exceeds
// 32767 - max(0, max score) may have overflowed: that pair is rescored at once
// by the same warp with the exact 32-bit code.  Cells past a query's rows,
// past a window's columns or on a half's idle passes score 0 and cannot raise
// the maximum (open, extend >= 0).
//
// Work: warps claim two entries of the 32-bit list's static part at a time;
// entries that are not banded pairs with int8 rows are left to the 32-bit
// kernel, which skips exactly the entries taken here (band16_takes).
#pragma once
#include "st_common.cuh"
#include "st_sw32.cuh"

namespace st {

constexpr uint32_t kBandNone = 0xFFFFFFFFu;

// A pair is scored here when it is banded and its rows fit int8 (the launch
// itself requires gap costs within the 16-bit range).
__device__ __forceinline__ bool band16_takes(const Sw32Params& prm, uint32_t p) {
  return prm.pair_radius[p] >= 0 && prm.prof.fits8[prm.pair_query[p]] != 0;
}

struct Band16Half {
  const uint8_t* t;    // target residues
  const int8_t* p8;    // int8 profile, residue-major [22][stride8]
  uint32_t stride8;
  int m, n, P;
  int64_t center, radius;
  int32_t thresh;      // headroom limit of the 16-bit cells
  bool on;
};

__device__ __forceinline__ Band16Half band16_half(const Sw32Params& prm, uint32_t p, bool* empty) {
  Band16Half h{};
  *empty = false;
  if (p == kBandNone) return h;
  const uint32_t q = prm.pair_query[p];
  const uint32_t tid = prm.pair_target[p];
  const int m = static_cast<int>(prm.prof.qlen[q]);
  const int n = static_cast<int>(prm.db.length[tid]);
  h.center = prm.pair_center[p];
  h.radius = prm.pair_radius[p];
  // columns that can hold band cells (as the 32-bit kernel)
  const int64_t c_lo = i64max(0, h.center - h.radius);
  const int64_t c_hi = i64min(n, static_cast<int64_t>(m) - 1 + h.center + h.radius + 1);
  if (m == 0 || n == 0 || c_hi <= c_lo) {
    *empty = true;
    return h;
  }
  h.t = prm.db.arena + prm.db.offset[tid];
  h.p8 = prm.prof.p8[q];
  h.stride8 = prm.prof.stride8[q];
  h.m = m;
  h.n = n;
  h.P = (m + kSw32Rows - 1) / kSw32Rows;
  h.thresh = 32767 - prm.prof.max_score[q];
  h.on = true;
  return h;
}

// Band window of pass p: the columns [cs, cs + ws) that hold band cells of rows
// [256p, 256p + 256) (clipped to the target; empty past the half's passes).
__device__ __forceinline__ void band16_win(const Band16Half& h, int p, int& cs, int& ws) {
  if (!h.on || p >= h.P) {
    cs = 0;
    ws = 0;
    return;
  }
  const int64_t r0 = static_cast<int64_t>(p) * kSw32Rows;
  const int64_t a = i64min(i64max(0, r0 + h.center - h.radius), h.n);
  const int64_t b = i64max(i64min(h.n, r0 + kSw32Rows - 1 + h.center + h.radius + 1), a);
  cs = static_cast<int>(a);
  ws = static_cast<int>(b - a);
}

// Band rows among the lane's 8 rows at absolute column a: an 8-bit mask, bit k
// set when row0 + k is within the band.
__device__ __forceinline__ uint32_t band16_rows(const Band16Half& h, int a, int row0) {
  if (!h.on) return 0;
  const int64_t base = static_cast<int64_t>(a) - row0 - h.center;
  const int64_t lo = base - h.radius, hi = base + h.radius;  // band rows: lo <= k <= hi
  if (hi < 0 || lo > 7) return 0;
  const int l = static_cast<int>(i64max(lo, 0)), u = static_cast<int>(i64min(hi, 7));
  return (0xFFu >> (7 - u)) & (0xFFu << l);
}

// Four mask bits -> four bytes 0x00 / 0xFF.
__device__ __forceinline__ uint32_t band16_bytes(uint32_t nib) {
  return ((nib * 0x00204081u) & 0x01010101u) * 0xFFu;
}

// This lane's 8 int8 scores of residue r at rows row0 .. row0 + 7 of one half
// (zero past the query: rows from m are never loaded).
__device__ __forceinline__ uint2 band16_scores(const Band16Half& h, uint32_t r, int row0) {
  if (!h.on || row0 >= h.m) return make_uint2(0u, 0u);
  return __ldg(reinterpret_cast<const uint2*>(h.p8 + static_cast<size_t>(r) * h.stride8 + row0));
}

// Each pass streams only its own band window (a 256-row pass of a long query
// needs 256 + 2 radius columns, not the whole pair's m + 2 radius).  The bottom
// row of a pass goes to the scratch line by absolute target column, per half:
// half A's (H, F) in the .x word of entry a, half B's in the .y word.  Pass p + 1
// reads column a of it if pass p wrote it; a column right of pass p's window is
// outside the band of pass p's last row (H = 0, F = -infinity, so its successor
// starts from -open).  Columns left of a pass's window are outside the band of
// all its rows, except the diagonal predecessor of the pass's first row, which
// lane 0 takes from the line too.  Lane 0 reads column a of pass p + 1 at step
// (p + 1) W + (a - cs_{p+1}); the last lane wrote it at step
// p W + (a - cs_p) + 31, earlier when W >= (cs_{p+1} - cs_p) + 32.
__device__ __forceinline__ void band16_couple(const Sw32Params& prm, uint32_t pA, uint32_t pB, int2* bnd_) {
  constexpr int G = kSw32G, R = kSw32R;
  const int lane = threadIdx.x & 31;
  const uint32_t FULL = 0xFFFFFFFFu;
  uint2* bnd = reinterpret_cast<uint2*>(bnd_);
  bool emptyA, emptyB;
  const Band16Half A = band16_half(prm, pA, &emptyA);
  const Band16Half B = band16_half(prm, pB, &emptyB);
  if (lane == 0) {  // a pair without band cells scores 0
    if (emptyA) {
      prm.scores[pA] = 0;
      if (prm.kernels) prm.kernels[pA] = 1u;
    }
    if (emptyB) {
      prm.scores[pB] = 0;
      if (prm.kernels) prm.kernels[pB] = 1u;
    }
  }
  if (!A.on && !B.on) return;
  const int P = max(A.on ? A.P : 0, B.on ? B.P : 0);
  // columns per pass: the widest window, and the shift of the windows plus a warp between passes
  int W = 0, shift = 0;
  for (int pp = 0; pp < P; ++pp) {
    int csA, wsA, csB, wsB;
    band16_win(A, pp, csA, wsA);
    band16_win(B, pp, csB, wsB);
    W = max(W, max(wsA, wsB));
    if (pp + 1 < P) {
      int nA, nwA, nB, nwB;
      band16_win(A, pp + 1, nA, nwA);
      band16_win(B, pp + 1, nB, nwB);
      if (pp + 1 < A.P) shift = max(shift, nA - csA);
      if (pp + 1 < B.P) shift = max(shift, nB - csB);
    }
  }
  if (P > 1) W = max(W, shift + G);
  const uint32_t MOPEN = pk_splat(-prm.open);
  const uint32_t MEXT = pk_splat(-prm.ext);
  const uint32_t E0 = MOPEN, F0 = MOPEN;  // first column / first row, and after a band reset
  const uint32_t F0h = F0 & 0xFFFFu;

  uint32_t Hp[R], E[R];
#pragma unroll
  for (int k = 0; k < R; ++k) {
    Hp[k] = 0;
    E[k] = E0;
  }
  uint32_t best = 0, hup_prev = 0, h_bot = 0, f_out = F0;
  int c = -lane;
  int pass = 0;
  int csA, wsA, csB, wsB;  // this lane's pass's windows
  band16_win(A, 0, csA, wsA);
  band16_win(B, 0, csB, wsB);
  // residue of a half at column c of a window (the sentinel past the window)
  auto res_at = [&](const Band16Half& h, int cs, int ws, int cc) -> uint32_t {
    if (cc >= ws) return kSentinel;
    return min(static_cast<uint32_t>(__ldg(h.t + cs + cc)), static_cast<uint32_t>(kSentinel));
  };
  // Software pipeline (as the 32-bit kernel): this step's residues and scores were loaded during the step
  // before; a lane's next residues are the ones its upper neighbour uses now.  Residues travel as one word:
  // half A in byte 0, half B in byte 1.  Lane 0 reads its columns two steps ahead: (c2, p2) and the windows
  // of pass p2.
  uint32_t res = kSentinel | (kSentinel << 8), q1 = kSentinel | (kSentinel << 8);
  int c2 = 2, p2 = 0;
  while (c2 >= W) {
    c2 -= W;
    ++p2;
  }
  int cs2A, ws2A, cs2B, ws2B;
  band16_win(A, p2, cs2A, ws2A);
  band16_win(B, p2, cs2B, ws2B);
  if (lane == 0) {
    res = res_at(A, csA, wsA, 0) | (res_at(B, csB, wsB, 0) << 8);
    const int c1 = 1 < W ? 1 : 0, p1 = 1 < W ? 0 : 1;
    int a1, w1, b1, v1;
    band16_win(A, p1, a1, w1);
    band16_win(B, p1, b1, v1);
    q1 = res_at(A, a1, w1, c1) | (res_at(B, b1, v1, c1) << 8);
  }
  uint2 sa = band16_scores(A, res & 0xFFu, lane * R);
  uint2 sb = band16_scores(B, res >> 8, lane * R);
  const int steps = P * W + G - 1;

  for (int s = 0; s < steps; ++s) {
    uint32_t hin = __shfl_up_sync(FULL, h_bot, 1);
    uint32_t fin = __shfl_up_sync(FULL, f_out, 1);
    uint32_t rn = __shfl_up_sync(FULL, res, 1);
    if (lane == 0) {
      // the previous pass's bottom row at this column, per half (or a fresh boundary)
      uint32_t hA = 0, fA = F0h, hB = 0, fB = F0h;
      if (pass > 0 && pass < P) {
        int pcs, pws;
        if (c < wsA && pass < A.P) {
          band16_win(A, pass - 1, pcs, pws);
          const int a = csA + c;
          if (a >= pcs && a < pcs + pws) {
            const uint32_t v = bnd[a].x;
            hA = v & 0xFFFFu;
            fA = v >> 16;
          }
        }
        if (c < wsB && pass < B.P) {
          band16_win(B, pass - 1, pcs, pws);
          const int a = csB + c;
          if (a >= pcs && a < pcs + pws) {
            const uint32_t v = bnd[a].y;
            hB = v & 0xFFFFu;
            fB = v >> 16;
          }
        }
      }
      hin = hA | (hB << 16);
      fin = fA | (fB << 16);
      rn = q1;
      q1 = res_at(A, cs2A, ws2A, c2) | (res_at(B, cs2B, ws2B, c2) << 8);
      if (++c2 == W) {
        c2 = 0;
        ++p2;
        band16_win(A, p2, cs2A, ws2A);
        band16_win(B, p2, cs2B, ws2B);
      }
    }
    int cn = c + 1, pn = pass;
    if (cn == W) {
      cn = 0;
      ++pn;
    }
    const int rown = (pn < P ? pn : P - 1) * G * R + lane * R;
    const uint2 san = band16_scores(A, rn & 0xFFu, rown);
    const uint2 sbn = band16_scores(B, rn >> 8, rown);
    if (c == 0) {
#pragma unroll
      for (int k = 0; k < R; ++k) {
        Hp[k] = 0;
        E[k] = E0;
      }
      hup_prev = 0;
      if (lane == 0 && pass > 0 && pass < P) {
        // the diagonal predecessor of the pass's first row: column cs - 1 of the previous pass's last row
        uint32_t dA = 0, dB = 0;
        int pcs, pws;
        if (pass < A.P) {
          band16_win(A, pass - 1, pcs, pws);
          const int a = csA - 1;
          if (a >= pcs && a < pcs + pws) dA = bnd[a].x & 0xFFFFu;
        }
        if (pass < B.P) {
          band16_win(B, pass - 1, pcs, pws);
          const int a = csB - 1;
          if (a >= pcs && a < pcs + pws) dB = bnd[a].y & 0xFFFFu;
        }
        hup_prev = dA | (dB << 16);
      }
    }
    const int pp = pass < P ? pass : P - 1;
    const int row0 = pp * G * R + lane * R;
    // band masks of this step: bytes 0xFF for band rows, per half, then one prmt per cell pair
    const uint32_t ba = (c >= 0 && c < wsA) ? band16_rows(A, csA + c, row0) : 0u;
    const uint32_t bb = (c >= 0 && c < wsB) ? band16_rows(B, csB + c, row0) : 0u;
    const uint32_t ma0 = band16_bytes(ba & 0xFu), ma1 = band16_bytes(ba >> 4);
    const uint32_t mb0 = band16_bytes(bb & 0xFu), mb1 = band16_bytes(bb >> 4);
    const uint32_t wa[2] = {sa.x, sa.y}, wb[2] = {sb.x, sb.y};
    uint32_t hd = hup_prev;
    uint32_t F = fin;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const uint32_t S = prmt(wa[k >> 2], wb[k >> 2], sel_pair(k & 3));
      const uint32_t M = prmt(k < 4 ? ma0 : ma1, k < 4 ? mb0 : mb1, static_cast<uint32_t>((k & 3) | ((k & 3) << 4) |
                                                                                      ((4 + (k & 3)) << 8) |
                                                                                      ((4 + (k & 3)) << 12)));
      const uint32_t t = pk_addmax(hd, S, E[k]);
      const uint32_t H = pk_max_relu(t, F) & M;  // out of the band (or of the window): H = 0
      best = pk_max(best, H);
      const uint32_t Ho = pk_add(H, MOPEN);
      // out of the band: E and F of the cell are minus infinity, so their successors start from -open
      E[k] = (pk_addmax(E[k], MEXT, Ho) & M) | (E0 & ~M);
      F = (pk_addmax(F, MEXT, Ho) & M) | (F0 & ~M);
      hd = Hp[k];
      Hp[k] = H;
    }
    hup_prev = hin;
    h_bot = Hp[R - 1];
    f_out = F;
    if (lane == G - 1 && c >= 0) {
      if (pass + 1 < A.P && c < wsA) bnd[csA + c].x = (h_bot & 0xFFFFu) | (f_out << 16);
      if (pass + 1 < B.P && c < wsB) bnd[csB + c].y = (h_bot >> 16) | (f_out & 0xFFFF0000u);
    }
    if (cn == 0 && pn != pass) {  // the next pass's windows
      band16_win(A, pn, csA, wsA);
      band16_win(B, pn, csB, wsB);
    }
    c = cn;
    pass = pn;
    res = rn;
    sa = san;
    sb = sbn;
    __syncwarp();
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = pk_max(best, __shfl_xor_sync(FULL, best, o));
  const int32_t bA = pk_lo(best), bB = pk_hi(best);
  // past the headroom: rescored exactly by the 32-bit code (the scratch line is free again)
  if (A.on) {
    if (bA > A.thresh) {
      sw32_pair<kSw32Score>(prm, pA, bnd_);
    } else if (lane == 0) {
      prm.scores[pA] = bA;
      if (prm.kernels) prm.kernels[pA] = 1u;
    }
  }
  if (B.on) {
    if (bB > B.thresh) {
      sw32_pair<kSw32Score>(prm, pB, bnd_);
    } else if (lane == 0) {
      prm.scores[pB] = bB;
      if (prm.kernels) prm.kernels[pB] = 1u;
    }
  }
}

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) sw16_band_kernel(const Sw32Params prm) {
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int2* bnd = prm.scratch + static_cast<size_t>(blockIdx.x * WARPS + warp) * prm.scratch_stride;
  const uint32_t n = prm.n_static;
  for (;;) {
    uint32_t w = 0;
    if (lane == 0) w = atomicAdd(prm.work_counter, 2u);
    w = __shfl_sync(0xFFFFFFFFu, w, 0);
    if (w >= n) break;
    const uint32_t a = prm.list[w];
    const uint32_t b = w + 1 < n ? prm.list[w + 1] : kBandNone;
    const uint32_t pA = band16_takes(prm, a) ? a : kBandNone;
    const uint32_t pB = (b != kBandNone && band16_takes(prm, b)) ? b : kBandNone;
    if (pA == kBandNone && pB == kBandNone) continue;
    band16_couple(prm, pA, pB, bnd);
  }
}

}  // namespace st
