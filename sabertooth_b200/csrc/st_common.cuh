// Shared device helpers: packed 16-bit cell arithmetic (DPX), byte permutes,
// constants of the residue alphabet and device-side data layouts.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace st {

// Residue alphabet: codes 0..20 score through the rows; every code >= 21 scores
// 0 (reference src/align.rs:180-186, src/simd.rs:367-368).  On the device all
// codes are clamped to kSentinel so profile lookups stay in a 22-row table
// whose last row is zero.
constexpr int kAlpha = 21;
constexpr int kProfRows = 22;
constexpr uint8_t kSentinel = 21;

// i32::MIN / 4, the "minus infinity" of the reference's scalar kernels
// (src/simd.rs:354, src/align.rs:287).
constexpr int32_t kNeg32 = INT32_MIN / 4;

// ---- packed s16x2 cells ---------------------------------------------------
// Low half = alignment A, high half = alignment B.  Every op is lane-wise with
// no carry between halves; adds wrap (they do not saturate), so the 16-bit
// kernel bounds every H by an explicit headroom test instead.
__device__ __forceinline__ uint32_t pk_addmax(uint32_t a, uint32_t b, uint32_t c) {
  return __viaddmax_s16x2(a, b, c);  // max(a + b, c)
}
__device__ __forceinline__ uint32_t pk_max_relu(uint32_t a, uint32_t b) {
  return __vimax_s16x2_relu(a, b);  // max(a, b, 0)
}
__device__ __forceinline__ uint32_t pk_max(uint32_t a, uint32_t b) { return __vmaxs2(a, b); }
__device__ __forceinline__ uint32_t pk_add(uint32_t a, uint32_t b) { return __vadd2(a, b); }

__host__ __device__ constexpr uint32_t pk_splat(int32_t v) {
  return (static_cast<uint32_t>(static_cast<uint16_t>(static_cast<int16_t>(v)))) |
         (static_cast<uint32_t>(static_cast<uint16_t>(static_cast<int16_t>(v))) << 16);
}
__device__ __forceinline__ int32_t pk_lo(uint32_t v) { return static_cast<int16_t>(v & 0xFFFFu); }
__device__ __forceinline__ int32_t pk_hi(uint32_t v) { return static_cast<int16_t>(v >> 16); }

// prmt.b32 in its default mode: selector bit 3 of each nibble replicates the
// sign of the selected byte, which sign-extends an int8 score into 16 bits.
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
  return d;
}
// Selector building {sext(a.byte[k]), sext(b.byte[k])} as an s16x2 pair.
__host__ __device__ constexpr uint32_t sel_pair(int k) {
  return static_cast<uint32_t>(k) | (static_cast<uint32_t>(k | 8) << 4) | (static_cast<uint32_t>(4 + k) << 8) |
         (static_cast<uint32_t>((4 + k) | 8) << 12);
}

// Wrapping 32-bit arithmetic (the reference's release build wraps on overflow).
__device__ __forceinline__ int32_t wadd(int32_t a, int32_t b) {
  return static_cast<int32_t>(static_cast<uint32_t>(a) + static_cast<uint32_t>(b));
}
__device__ __forceinline__ int32_t wsub(int32_t a, int32_t b) {
  return static_cast<int32_t>(static_cast<uint32_t>(a) - static_cast<uint32_t>(b));
}

__host__ __device__ __forceinline__ int64_t i64max(int64_t a, int64_t b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ int64_t i64min(int64_t a, int64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ uint64_t u64min(uint64_t a, uint64_t b) { return a < b ? a : b; }

// ---- device layouts --------------------------------------------------------
// Target database: every sequence starts on a 16-byte boundary of one arena and
// is followed by sentinel bytes up to the next multiple of 16 (plus 16 spare
// sentinel bytes at the arena end), so 16-byte vector loads never cross into
// the next sequence.
struct DeviceDb {
  const uint8_t* arena;
  const uint64_t* offset;  // start of sequence s (multiple of 16)
  const uint32_t* length;  // residues of sequence s
  uint32_t n_seqs;
};

// Query profiles, residue-major: profile q, residue r, row i at
//   p8 [q][r * stride8[q]  + i]   (int8; all zero unless every score fits int8)
//   p32[q][r * stride32[q] + i]   (int32, always)
// Row kAlpha (= 21) is all zero; rows i >= m are zero up to the stride.
// stride8 is a multiple of 16, stride32 a multiple of 256 (one 32-bit pass).
struct DeviceProfiles {
  const int8_t* const* p8;
  const int32_t* const* p32;
  const uint32_t* stride8;
  const uint32_t* stride32;
  const uint32_t* qlen;
  const int32_t* max_score;  // max(0, largest score of the profile)
  const uint8_t* fits8;      // 1 when every score is within int8
};

}  // namespace st
