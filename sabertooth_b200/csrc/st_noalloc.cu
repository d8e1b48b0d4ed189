// st_sw_score_noalloc: exact Smith-Waterman-Gotoh score of one pair over
// caller-owned device buffers, with no device memory allocation at all.
//
// Who needs this: callers that must not call cudaMalloc / cudaFree.  Typical
// ones are code that runs while a CUDA stream is being captured into a graph
// (CUDA treats allocation as unsafe during a global-mode capture), latency-bound
// serving threads that cannot pay for the implicit device synchronisation of
// cudaFree, and host processes whose device memory is owned by another
// allocator (a framework's caching pool, a fixed arena) where an extra raw
// allocation would fail or fragment it.  Such callers hand in device
// pointers they already own and get the score written to another.
//
// The kernel is the exact 32-bit recurrence of the context-based 32-bit
// kernel (literal Gotoh in wrapping int32, i32::MIN/4 as minus infinity, so it
// matches the reference's scalar path for any gap costs), reading the score
// rows in their int32 [m][21] row-major form.  Its only scratch — the bottom
// row (H, F) of each 256-row pass over the query, read back by the next pass —
// lives in the file-scope device array below instead of an allocation.
//
// The array is a fixed 512 KiB (kNoAllocMaxCols entries of int2) held by every
// GPU that loads this library until the process exits; it bounds the target
// length to kNoAllocMaxCols residues.  All calls on a device share it and it
// keeps whatever the last call wrote.  Nothing in it has to start at zero: a
// call reads an entry back only after writing it in the same call (a query of
// more than 256 rows streams at least 32 columns per pass, so the boundary of
// a column is written before the next pass reaches it).  Calls whose
// kernels overlap on the GPU (for example on two streams without an event
// between them) race on the array and may return wrong scores; issue them on
// one stream or order them.
//
// Set-up: the first call on a device looks up the device address of the array
// (cudaGetSymbolAddress, with that device current) and caches it; later calls
// only launch.  Make that first call before any stream capture begins (a warm-up
// call with n = 0 is enough).  The cache lives for the process: after a
// cudaDeviceReset the device holds a new copy of the array at an address this
// cache does not know, so a device that was reset must not be used here again.
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/sabertooth_b200.h"
#include "st_common.cuh"

namespace {

using namespace st;

constexpr uint32_t kNoAllocMaxCols = 65536;
constexpr uint32_t kNoAllocMaxRows = 1u << 20;
constexpr int kMaxDevices = 64;

// boundary rows of the passes: (H, F) per target column
static __device__ __align__(256) int2 g_noalloc_scratch[kNoAllocMaxCols];

constexpr int G = 32;  // lanes of the one warp
constexpr int R = 8;   // query rows per lane; one pass covers G * R = 256 rows

__global__ void __launch_bounds__(32) sw_noalloc_kernel(const int32_t* __restrict__ rows, uint32_t m_,
                                                        const uint8_t* __restrict__ t, uint32_t n_, int32_t open,
                                                        int32_t ext, int2* __restrict__ bnd, int32_t* out) {
  const int lane = threadIdx.x & 31;
  const uint32_t FULL = 0xFFFFFFFFu;
  const int m = static_cast<int>(m_), n = static_cast<int>(n_);
  if (m == 0 || n == 0) {
    if (lane == 0) *out = 0;
    return;
  }
  const int P = (m + G * R - 1) / (G * R);
  // Columns streamed per pass: lane 0 reads column c's boundary of pass p at
  // step p*W + c, and lane G-1 wrote it at step (p-1)*W + c + G-1, so W must be
  // at least G.  Against a target shorter than G, a multi-pass query streams
  // idle columns [n, G) after the real ones; they carry the sentinel residue,
  // never count toward the maximum, never touch the boundary array, and the
  // state they leave is reset when the next pass starts at column 0.
  const int W = P > 1 ? max(n, G) : n;
  const int32_t E0 = max(wsub(0, open), wsub(kNeg32, ext));  // first-column E, first-row F
  const int32_t F0 = E0;
  int32_t Hp[R], E[R];
#pragma unroll
  for (int k = 0; k < R; ++k) {
    Hp[k] = 0;
    E[k] = E0;
  }
  int32_t best = 0, hup_prev = 0, h_bot = 0, f_out = F0;
  uint32_t res = kSentinel;
  int c = -lane;  // this lane's column (negative: not started)
  int pass = 0;
  uint32_t nxt = kSentinel;
  if (lane == 0) nxt = min(static_cast<uint32_t>(t[0]), static_cast<uint32_t>(kSentinel));
  const int steps = P * W + G - 1;
  for (int s = 0; s < steps; ++s) {
    int32_t hin = __shfl_up_sync(FULL, h_bot, 1);
    int32_t fin = __shfl_up_sync(FULL, f_out, 1);
    uint32_t rin = __shfl_up_sync(FULL, res, 1);
    if (lane == 0) {
      if (pass < P) {
        rin = nxt;
        int cn = c + 1;
        const bool last = (cn == W);
        if (last) cn = 0;
        nxt = ((last && pass + 1 >= P) || cn >= n) ? kSentinel
                                                   : min(static_cast<uint32_t>(t[cn]), static_cast<uint32_t>(kSentinel));
        if (pass > 0 && c < n) {
          const int2 bv = bnd[c];
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
    const bool live = (c >= 0) && (c < n) && (pass < P);
    int32_t hd = hup_prev;
    int32_t F = fin;
    int32_t lmax = 0;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int row = row0 + k;
      const int32_t S = (row < m && res < static_cast<uint32_t>(kAlpha)) ? rows[static_cast<size_t>(row) * kAlpha + res] : 0;
      const int32_t tt = max(wadd(hd, S), E[k]);
      const int32_t H = max(max(tt, F), 0);
      const int32_t Ho = wsub(H, open);
      E[k] = max(wsub(E[k], ext), Ho);
      F = max(wsub(F, ext), Ho);
      if (row < m) lmax = max(lmax, H);
      hd = Hp[k];
      Hp[k] = H;
    }
    if (live) best = max(best, lmax);
    hup_prev = hin;
    h_bot = Hp[R - 1];
    f_out = F;
    if (lane == G - 1 && pass + 1 < P && c >= 0 && c < n) bnd[c] = make_int2(h_bot, f_out);
    if (++c == W) {
      c = 0;
      ++pass;
    }
    __syncwarp();
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(FULL, best, o));
  if (lane == 0) *out = best;
}

std::mutex g_addr_mu;
int2* g_addr[kMaxDevices] = {};

}  // namespace

// Reports through st_last_error(), as every other entry point (defined in st_runtime.cu).
void st_internal_set_error(const char* msg);

static int noalloc_fail(int code, const char* msg) {
  st_internal_set_error(msg);
  return code;
}

extern "C" int st_sw_score_noalloc(const int32_t* d_rows, uint32_t m, const uint8_t* d_target, uint32_t n,
                                   int32_t open, int32_t ext, int32_t* d_score, void* stream) {
  if (!d_score || (m && !d_rows) || (n && !d_target))
    return noalloc_fail(ST_EINVAL, "st_sw_score_noalloc: null device pointer");
  if (n > kNoAllocMaxCols)
    return noalloc_fail(ST_EINVAL,
                        "st_sw_score_noalloc: the target is longer than the 65536 residues its static scratch holds");
  if (m > kNoAllocMaxRows)
    return noalloc_fail(ST_EINVAL, "st_sw_score_noalloc: the query is longer than 2^20 rows");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return noalloc_fail(ST_ECUDA, "st_sw_score_noalloc: no current CUDA device");
  int2* scratch = nullptr;
  {
    // first call on this device: resolve the device address of the static scratch array
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        char buf[256];
        snprintf(buf, sizeof(buf), "st_sw_score_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return noalloc_fail(ST_ECUDA, buf);
      }
      g_addr[dev] = static_cast<int2*>(p);
    }
    scratch = g_addr[dev];
  }
  sw_noalloc_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(d_rows, m, d_target, n, open, ext, scratch,
                                                                     d_score);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char buf[256];
    snprintf(buf, sizeof(buf), "st_sw_score_noalloc: launch failed: %s", cudaGetErrorString(e));
    return noalloc_fail(ST_ECUDA, buf);
  }
  return ST_OK;
}
