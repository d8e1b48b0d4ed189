// Background targets of the per-profile calibration (calibrate_profile,
// reference src/evalue.rs:714-748) generated on the device.
//
// Sample i draws from SplitMix64 seeded by stream_seed(seed, 0xBEEF, i)
// (src/evalue.rs:53-81): the first draw picks its length (on the host, which
// needs the lengths for the layout), draw k + 2 its residue k: the state of
// SplitMix64 after j draws is seed + j * golden, so residue k is a pure
// function of (state after the length draw, k) and every residue is generated
// by its own thread.  A residue is the first of the 20 background classes whose
// cumulative probability exceeds next_f64() (BackgroundSampler::sample,
// :101-109); the uniform (x >> 11) / 2^53 and the comparisons are exact in
// binary64, so the sequences are the reference's bit for bit.
#pragma once
#include "st_common.cuh"

namespace st {

constexpr uint64_t kSplitMixGamma = 0x9E3779B97F4A7C15ull;

__host__ __device__ __forceinline__ uint64_t splitmix_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct CalibGen {
  const uint64_t* state;   // per sample: SplitMix64 state after the length draw
  const uint64_t* offset;  // per sample: arena offset (multiple of 16)
  const uint32_t* length;  // per sample: residues
  uint8_t* arena;
  double cum[20];          // cumulative background probabilities, cum[19] = 1
};

__global__ void __launch_bounds__(256) calib_targets_kernel(const CalibGen g) {
  const uint32_t i = blockIdx.x;
  const uint64_t s = g.state[i];
  const uint32_t n = g.length[i];
  uint8_t* out = g.arena + g.offset[i];
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
    const uint64_t z = splitmix_mix(s + (static_cast<uint64_t>(k) + 1) * kSplitMixGamma);
    const double u = static_cast<double>(z >> 11) / 9007199254740992.0;  // 2^53
    uint8_t r = 19;
#pragma unroll
    for (int j = 19; j >= 0; --j)
      if (u < g.cum[j]) r = static_cast<uint8_t>(j);
    out[k] = r;
  }
}

}  // namespace st
