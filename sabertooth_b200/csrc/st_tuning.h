// Tile-class selection for the packed 16-bit kernel: lanes per alignment (G)
// and query rows per lane (R) per length bin.  A table filled by the autotuner
// (st_autotune) takes precedence; empty entries fall back to a cost model of
// the wavefront: a warp task streams P * ncols + G - 1 steps, each costing
// about R row-updates plus a fixed per-step overhead, for 64 / G targets.
#pragma once
#include <cstdint>

constexpr int kTuneMBins = 10;  // query length: <=32, <=64, ..., <=8192, >8192
constexpr int kTuneNBins = 8;   // mean target length: <=64, <=128, ..., <=4096, >4096
constexpr int kMaxTileClasses = 16;

struct Tuning {
  int table[kTuneMBins][kTuneNBins];  // class index, -1 = cost model
  double step_overhead;               // per-step overhead in row-update units
};

int st_tuning_num_classes();
void st_tuning_class_shape(int c, int* G, int* R, int* C);

inline int tune_mbin(uint32_t m) {
  int b = 0;
  uint32_t lim = 32;
  while (b < kTuneMBins - 1 && m > lim) {
    ++b;
    lim <<= 1;
  }
  return b;
}

inline int tune_nbin(uint32_t n) {
  int b = 0;
  uint32_t lim = 64;
  while (b < kTuneNBins - 1 && n > lim) {
    ++b;
    lim <<= 1;
  }
  return b;
}

inline void tuning_defaults(Tuning* t) {
  for (int i = 0; i < kTuneMBins; ++i)
    for (int j = 0; j < kTuneNBins; ++j) t->table[i][j] = -1;
  t->step_overhead = 8.0;
}

// Estimated cost of scoring one query (m rows) against targets of mean length n in class c:
// a warp streams P * ncols / C steps per warp task of 64/G targets, each step costing R*C
// row updates plus a per-step overhead; a lone alignment also pays the wavefront ramp.
inline double tune_cost(const Tuning* t, int c, uint32_t m, uint32_t n, bool single) {
  int G, R, C;
  st_tuning_class_shape(c, &G, &R, &C);
  const uint32_t rows = static_cast<uint32_t>(G * R);
  const uint32_t P = (m + rows - 1) / rows;
  if (22.0 * P * rows > 216.0 * 1024) return 1e300;  // profile does not fit shared memory
  double ncols = n < 32 ? 32.0 : static_cast<double>((n + 15) & ~15u);
  if (P > 1 && ncols < C * G) ncols = ((C * G + 15) / 16) * 16.0;
  const double steps = P * ncols / C;
  const double per_step = R * C + t->step_overhead;
  if (single) return (steps + G - 1) * per_step;
  return steps * per_step * G / 64.0;
}

inline int tuning_model_pick(const Tuning* t, uint32_t m, uint32_t n, bool single) {
  int best = 0;
  double bc = 1e301;
  for (int c = 0; c < st_tuning_num_classes(); ++c) {
    const double v = tune_cost(t, c, m, n, single);
    if (v < bc) {
      bc = v;
      best = c;
    }
  }
  return best;
}

inline int tuning_pick(const Tuning* t, uint32_t m, uint32_t mean_n) {
  const int c = t->table[tune_mbin(m)][tune_nbin(mean_n)];
  if (c >= 0 && c < st_tuning_num_classes() && tune_cost(t, c, m, mean_n, false) < 1e300) return c;
  return tuning_model_pick(t, m, mean_n, false);
}

// Within the chosen class's family (same lanes per alignment G and columns per
// step C), the rows per lane R that best fits this query's length.
inline int tuning_refine(const Tuning* t, int c, uint32_t m, uint32_t n) {
  int G0, R0, C0;
  st_tuning_class_shape(c, &G0, &R0, &C0);
  int best = c;
  double bc = tune_cost(t, c, m, n, false);
  for (int k = 0; k < st_tuning_num_classes(); ++k) {
    int G, R, C;
    st_tuning_class_shape(k, &G, &R, &C);
    if (G != G0 || C != C0 || k == c) continue;
    const double v = tune_cost(t, k, m, n, false);
    if (v < bc * 0.97) {  // a clear win only: measured classes keep their edge
      bc = v;
      best = k;
    }
  }
  return best;
}

inline int tuning_pick_single(const Tuning* t, uint32_t m, uint32_t n) { return tuning_model_pick(t, m, n, true); }
