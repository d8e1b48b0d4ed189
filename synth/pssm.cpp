// Input generation (synthetic workloads, golden fixtures): PSSM construction
// from a numeric MSA, restating
// the reference's Profile::from_numeric_msa (src/profile.rs:90-341) step for
// step in single precision and in the reference's operation order, so the
// resulting int8 PSSM is the one the reference would build.  Compiled without
// floating-point contraction (no fused multiply-add), as the reference.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "pssm.h"

namespace {

constexpr int kAA = 20;         // PROFILE_AA_SIZE, src/alphabet.rs:17
constexpr uint8_t kGap = 0xFF;  // GAP, src/alphabet.rs:36

// src/profile.rs:219-255
void sequence_weights(const uint8_t* msa, uint32_t n, uint32_t L, std::vector<float>& w) {
  w.assign(n, 1e-6f);
  std::vector<uint32_t> nres(n, 0);
  for (uint32_t k = 0; k < n; ++k) {
    uint32_t nr = 0;
    for (uint32_t p = 0; p < L; ++p)
      if (msa[static_cast<size_t>(k) * L + p] != kGap) ++nr;
    nres[k] = nr;
  }
  int32_t nl[kAA];
  for (uint32_t pos = 0; pos < L; ++pos) {
    for (int a = 0; a < kAA; ++a) nl[a] = 0;
    for (uint32_t k = 0; k < n; ++k) {
      const uint8_t c = msa[static_cast<size_t>(k) * L + pos];
      if (c < kAA) nl[c] += 1;
    }
    int32_t distinct = 0;
    for (int a = 0; a < kAA; ++a)
      if (nl[a] > 0) ++distinct;
    if (distinct == 0) continue;
    for (uint32_t k = 0; k < n; ++k) {
      const uint8_t c = msa[static_cast<size_t>(k) * L + pos];
      if (c < kAA) {
        const float denom = static_cast<float>(nl[c]) * static_cast<float>(distinct) *
                            (static_cast<float>(nres[k]) + 30.0f);
        w[k] += 1.0f / denom;
      }
    }
  }
}

// src/profile.rs:344-358
void normalize_to_1(float* v, const double* bg) {
  float sum = 0.0f;
  for (int i = 0; i < kAA; ++i) sum += v[i];
  if (sum != 0.0f) {
    const float fac = 1.0f / sum;
    for (int i = 0; i < kAA; ++i) v[i] *= fac;
  } else if (bg) {
    for (int i = 0; i < kAA; ++i) v[i] = static_cast<float>(bg[i]);
  }
}

// src/profile.rs:258-301
void compute_neff(const std::vector<float>& freq, const std::vector<float>& w, const uint8_t* msa, uint32_t n,
                  uint32_t L, std::vector<float>& neff) {
  float neff_hmm = 0.0f;
  for (uint32_t pos = 0; pos < L; ++pos) {
    float sum = 0.0f;
    for (int a = 0; a < kAA; ++a) {
      const float f = freq[static_cast<size_t>(pos) * kAA + a];
      if (f > 1e-10f) sum -= f * log2f(f);
    }
    neff_hmm += exp2f(sum);
  }
  neff_hmm /= static_cast<float>(L > 0 ? L : 1);
  const float nlim = std::fmax(10.0f, neff_hmm + 1.0f);
  const float scale = log2f((nlim - neff_hmm) / (nlim - 1.0f));
  neff.assign(L, 0.0f);
  for (uint32_t pos = 0; pos < L; ++pos) {
    float w_m = -1.0f / static_cast<float>(n);
    for (uint32_t k = 0; k < n; ++k)
      if (msa[static_cast<size_t>(k) * L + pos] != kGap) w_m += w[k];
    neff[pos] = w_m < 0.0f ? 1.0f : nlim - (nlim - 1.0f) * exp2f(scale * w_m);
  }
}

inline int8_t round_clamp_i8(float val) {
  // src/profile.rs:335-337: round half away from zero, clamp, truncate (NaN -> 0)
  if (std::isnan(val)) return 0;
  float r = val < 0.0f ? val - 0.5f : val + 0.5f;
  if (r < -128.0f) r = -128.0f;
  if (r > 127.0f) r = 127.0f;
  return static_cast<int8_t>(static_cast<int>(r));
}

}  // namespace

extern "C" int st_pssm_from_msa(const uint8_t* msa, uint32_t n, uint32_t L, const float* r, const double* p_back,
                                float pca, float pcb, float score_bias, int8_t* pssm, float* neff_out) {
  if (n == 0 || L == 0 || !msa || !r || !p_back || !pssm) return -1;
  std::vector<float> w;
  sequence_weights(msa, n, L, w);
  float total = 0.0f;
  for (uint32_t k = 0; k < n; ++k) total += w[k];
  if (total > 0.0f) {
    for (uint32_t k = 0; k < n; ++k) w[k] = w[k] / total;
  } else {
    for (uint32_t k = 0; k < n; ++k) w[k] = 1.0f / static_cast<float>(n);
  }
  std::vector<float> freq(static_cast<size_t>(L) * kAA, 0.0f);
  for (uint32_t pos = 0; pos < L; ++pos) {
    float* f = &freq[static_cast<size_t>(pos) * kAA];
    for (uint32_t k = 0; k < n; ++k) {
      const uint8_t c = msa[static_cast<size_t>(k) * L + pos];
      if (c < kAA) f[c] += w[k];
    }
    normalize_to_1(f, p_back);
  }
  std::vector<float> neff;
  compute_neff(freq, w, msa, n, L, neff);
  std::vector<float> prob(static_cast<size_t>(L) * kAA, 0.0f);
  if (pca > 0.0f) {
    std::vector<float> g(static_cast<size_t>(L) * kAA, 0.0f);
    for (uint32_t pos = 0; pos < L; ++pos) {
      const size_t base = static_cast<size_t>(pos) * kAA;
      for (int a = 0; a < kAA; ++a) {
        float acc = 0.0f;
        for (int b = 0; b < kAA; ++b) acc += r[a * kAA + b] * freq[base + b];
        g[base + a] = acc;
      }
    }
    for (uint32_t pos = 0; pos < L; ++pos) {
      const size_t base = static_cast<size_t>(pos) * kAA;
      float tau = pca / (1.0f + neff[pos] / pcb);
      if (tau > 1.0f) tau = 1.0f;
      for (int a = 0; a < kAA; ++a) prob[base + a] = (1.0f - tau) * freq[base + a] + tau * g[base + a];
    }
  } else {
    prob = freq;
  }
  const float bit = 8.0f;  // PROFILE_BIT_FACTOR, src/profile.rs:28
  for (uint32_t pos = 0; pos < L; ++pos) {
    const size_t base = static_cast<size_t>(pos) * kAA;
    for (int a = 0; a < kAA; ++a) {
      const float p = prob[base + a];
      const float log_prob = log2f(p / static_cast<float>(p_back[a]));
      const float val = bit * log_prob + bit * score_bias;
      pssm[base + a] = round_clamp_i8(val);
    }
  }
  if (neff_out) std::memcpy(neff_out, neff.data(), L * sizeof(float));
  return 0;
}

extern "C" int st_pssm_batch(const uint8_t* msa, const uint64_t* msa_off, const uint32_t* n_rows,
                             const uint32_t* query_len, uint32_t n_msas, const float* r, const double* p_back,
                             float pca, float pcb, float score_bias, int8_t* pssm, const uint64_t* pssm_off,
                             int nthreads) {
  int err = 0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads > 0 ? nthreads : 1) reduction(| : err)
  for (int64_t k = 0; k < static_cast<int64_t>(n_msas); ++k) {
    err |= st_pssm_from_msa(msa + msa_off[k], n_rows[k], query_len[k], r, p_back, pca, pcb, score_bias,
                            pssm + pssm_off[k], nullptr) != 0;
  }
  return err ? -1 : 0;
}
