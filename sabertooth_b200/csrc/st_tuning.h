// Tile-class selection for the packed 16-bit kernel: lanes per alignment (G),
// query rows per lane (R) and columns per step (C).
//
// Batches: each query takes the class with the least estimated time, its
// streamed cells (padded rows x padded columns x slots, from its own target
// lengths) divided by the class's measured rate (streamed cells per second,
// calibrated by st_autotune; built-in B200 figures by default, 0 = class not
// considered).  A table entry per (query length, mean target length) bin, set
// by the caller, forces a class for that bin.
//
// Single alignments (the per-call path) use a model of the wavefront: a task
// streams P * ncols / C + G - 1 steps, each costing about R * C row updates
// plus a fixed per-step overhead.
#pragma once
#include <algorithm>
#include <cstdint>

constexpr int kTuneMBins = 10;  // query length: <=32, <=64, ..., <=8192, >8192
constexpr int kTuneNBins = 8;   // mean target length: <=64, <=128, ..., <=4096, >4096
constexpr int kMaxTileClasses = 32;

struct Tuning {
  int table[kTuneMBins][kTuneNBins];  // class index, -1 = rate model
  double step_overhead;               // per-step overhead in row-update units (single alignments)
  float rate[kMaxTileClasses];        // streamed cells per second / 1e12, per class; 0 = not used
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

// Rates measured on B200 (148 SMs, 1965 MHz), streamed cells per second / 1e12,
// with every query of the PSSM workload (4,000 queries of 50-2,000 rows, 1.2 M
// pairs, targets of 160 residues on average) forced into one class.
inline float tuning_default_rate(int G, int R, int C) {
  if (C != 4) return 0.0f;
  static const struct {
    int G, R;
    float rate;
  } kRates[] = {
      {4, 8, 3.826f}, {8, 8, 4.573f}, {16, 8, 4.578f}, {32, 8, 4.483f},
      {4, 12, 3.832f}, {8, 12, 4.817f}, {16, 12, 4.879f}, {32, 12, 4.665f},
      {4, 16, 3.986f}, {8, 16, 4.959f}, {16, 16, 5.011f}, {32, 16, 4.788f},
      {4, 20, 4.451f}, {8, 20, 5.240f}, {16, 20, 5.198f}, {32, 20, 5.069f},
      {4, 24, 4.680f}, {8, 24, 5.405f}, {16, 24, 5.399f}, {32, 24, 5.128f},
      {4, 28, 5.289f}, {8, 28, 5.362f}, {16, 28, 4.958f}, {4, 32, 5.194f},
      {8, 32, 5.233f}, {16, 32, 5.126f},
  };
  for (const auto& r : kRates)
    if (r.G == G && r.R == R) return r.rate;
  return 0.0f;
}

inline void tuning_defaults(Tuning* t) {
  for (int i = 0; i < kTuneMBins; ++i)
    for (int j = 0; j < kTuneNBins; ++j) t->table[i][j] = -1;
  t->step_overhead = 8.0;
  for (int c = 0; c < kMaxTileClasses; ++c) t->rate[c] = 0.0f;
  for (int c = 0; c < st_tuning_num_classes() && c < kMaxTileClasses; ++c) {
    int G, R, C;
    st_tuning_class_shape(c, &G, &R, &C);
    t->rate[c] = tuning_default_rate(G, R, C);
  }
}

// Streamed cells of one query (m rows) in class c over its targets' lengths,
// sorted longest first: warp tasks of 64/G targets stream the longest one's
// length rounded up to 4 columns (at least C*G columns when the query takes
// several passes).
inline double tune_streamed(int c, uint32_t m, const uint32_t* tlen_desc, size_t n) {
  int G, R, C;
  st_tuning_class_shape(c, &G, &R, &C);
  const uint32_t rows = static_cast<uint32_t>(G * R);
  const uint32_t P = (m + rows - 1) / rows;
  if (22.0 * P * rows > 216.0 * 1024) return 1e300;  // profile does not fit shared memory
  const uint32_t S = static_cast<uint32_t>(64 / G);
  uint32_t minc = 32;
  if (P > 1) minc = std::max<uint32_t>(minc, (static_cast<uint32_t>(C * G) + 15) & ~15u);
  double cols = 0;
  for (size_t w = 0; w < n; w += S) cols += std::max<uint32_t>(minc, (tlen_desc[w] + 3) & ~3u);
  return cols * S * P * rows;
}

// The class with the least estimated time for one query of a batch.
inline int tuning_pick_batch(const Tuning* t, uint32_t m, const uint32_t* tlen_desc, size_t n, uint32_t mean_n) {
  const int forced = t->table[tune_mbin(m)][tune_nbin(mean_n)];
  if (forced >= 0 && forced < st_tuning_num_classes() && tune_streamed(forced, m, tlen_desc, n) < 1e300) return forced;
  // classes with a rate first; if none of them stages this query, least streamed cells over all
  int best = -1;
  for (int pass = 0; pass < 2 && best < 0; ++pass) {
    double bt = 1e299;
    for (int c = 0; c < st_tuning_num_classes() && c < kMaxTileClasses; ++c) {
      if (pass == 0 && !(t->rate[c] > 0.0f)) continue;
      const double v = tune_streamed(c, m, tlen_desc, n) / (pass == 0 ? t->rate[c] : 1.0f);
      if (v < bt) {
        bt = v;
        best = c;
      }
    }
  }
  return best;
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

inline int tuning_pick_single(const Tuning* t, uint32_t m, uint32_t n) { return tuning_model_pick(t, m, n, true); }
