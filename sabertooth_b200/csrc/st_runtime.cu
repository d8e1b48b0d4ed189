// Runtime behind the C ABI (include/sabertooth_b200.h): context, device-resident
// target database and query profiles, the batch planner (length bins, tile
// classes, persistent-kernel work lists, CUDA-graph capture) and the plain
// per-call paths that replace the reference's QueryProfile::sw_score_with and
// ungapped::score_batch.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <shared_mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/sabertooth_b200.h"
#include "st_common.cuh"
#include "st_sw16.cuh"
#include "st_sw32.cuh"
#include "st_band16.cuh"
#include "st_tuning.h"
#include "st_ungapped.cuh"
#include "st_dplan.cuh"
#include "st_gate.cuh"
#include "st_calib.cuh"
#include "st_seed.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <cub/iterator/counting_input_iterator.cuh>
#include <cub/iterator/transform_input_iterator.cuh>

using namespace st;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define ST_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return fail(ST_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                       __FILE__, __LINE__);                                        \
  } while (0)

#define ST_TRY(expr)          \
  do {                        \
    int r_ = (expr);          \
    if (r_ != ST_OK) return r_; \
  } while (0)

extern "C" const char* st_last_error(void) { return g_last_error.c_str(); }

// Host phase tracing (ST_TRACE=1 in the environment): one line per phase on stderr.
#include <chrono>
static bool trace_on() {
  static const bool on = [] {
    const char* v = getenv("ST_TRACE");
    return v && v[0] && v[0] != '0';
  }();
  return on;
}
// A numeric setting from the environment, or the default.
static uint64_t env_u64(const char* name, uint64_t dflt) {
  const char* v = getenv(name);
  if (!v || !*v) return dflt;
  return strtoull(v, nullptr, 10);
}

// Traces a driver call of the memory helpers that took longer than a millisecond.
struct SlowCall {
  const char* what;
  size_t bytes;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  SlowCall(const char* w, size_t b) : what(w), bytes(b) {}
  ~SlowCall() {
    if (!trace_on()) return;
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (ms > 1.0) fprintf(stderr, "[st] slow %s %zu bytes %.3f ms\n", what, bytes, ms);
  }
};

struct TraceClock {
  const char* what;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  explicit TraceClock(const char* w) : what(w) {}
  void lap(const char* phase) {
    if (!trace_on()) return;
    const auto t1 = std::chrono::steady_clock::now();
    fprintf(stderr, "[st] %s %s %.3f ms\n", what, phase, std::chrono::duration<double, std::milli>(t1 - t0).count());
    t0 = t1;
  }
};

// Lets other translation units of the library report through st_last_error().
__attribute__((visibility("hidden"))) void st_internal_set_error(const char* msg) { g_last_error = msg; }

// ---------------------------------------------------------------------------
// device memory with budget accounting
// ---------------------------------------------------------------------------
struct MemTracker {
  size_t used = 0;
  size_t budget = 0;  // 0 = unlimited
};

struct DevMem {
  void* p = nullptr;
  size_t bytes = 0;
  MemTracker* mt = nullptr;
  DevMem() = default;
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
  DevMem(DevMem&& o) noexcept { *this = std::move(o); }
  DevMem& operator=(DevMem&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      bytes = o.bytes;
      mt = o.mt;
      o.p = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DevMem() { release(); }
  void release() {
    if (p) {
      SlowCall sc("cudaFree", bytes);
      cudaFree(p);
      if (mt) mt->used -= bytes;
    }
    p = nullptr;
    bytes = 0;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

static int dev_alloc(MemTracker* mt, DevMem& m, size_t bytes) {
  m.release();
  if (bytes == 0) bytes = 16;
  if (mt->budget && mt->used + bytes > mt->budget)
    return fail(ST_ENOMEM, "device memory budget exceeded: %zu used + %zu requested > %zu budget", mt->used,
                bytes, mt->budget);
  cudaError_t e;
  {
    SlowCall sc("cudaMalloc", bytes);
    e = cudaMalloc(&m.p, bytes);
  }
  if (e != cudaSuccess) {
    m.p = nullptr;
    return fail(ST_ENOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  m.bytes = bytes;
  m.mt = mt;
  mt->used += bytes;
  return ST_OK;
}

// pinned host staging buffer that only grows
struct Pinned {
  void* p = nullptr;
  size_t bytes = 0;
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
  // Grows by at least half the current size, to a size class (2^k times 1, 1.25,
  // 1.5 or 1.75): freeing pinned memory waits for the whole device, so a buffer
  // that follows slowly growing batches should reallocate rarely.
  int reserve(size_t n) {
    if (n <= bytes) return ST_OK;
    const size_t target = std::max<size_t>(n, bytes + bytes / 2);
    size_t cls = 1 << 20;
    while (cls < target) cls <<= 1;
    size_t want = cls;
    for (size_t k = 5; k <= 8; ++k)
      if (cls / 8 * k >= target) {
        want = cls / 8 * k;
        break;
      }
    SlowCall sc("pinned regrow", want);
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    ST_CUDA(cudaMallocHost(&p, want));
    bytes = want;
    return ST_OK;
  }
  template <class T>
  T* as(size_t off = 0) const {
    return reinterpret_cast<T*>(static_cast<char*>(p) + off);
  }
};

static inline size_t up16(size_t x) { return (x + 15) & ~static_cast<size_t>(15); }

static bool host_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // not a CUDA-known pointer: pageable
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

static inline size_t up4(size_t x) { return (x + 3) & ~static_cast<size_t>(3); }
static inline size_t up256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// ---------------------------------------------------------------------------
// kernel classes
// ---------------------------------------------------------------------------
constexpr int kWarps16 = 8;
constexpr int kWarps32 = 4;
constexpr int kMaxSmem = 226 * 1024;  // dynamic shared memory per CTA (the 227 KB opt-in less room for static shared)

using Sw16Fn = void (*)(const Sw16Params);

struct Sw16Class {
  int G, R, C, W;  // lanes per alignment, rows per lane, columns per step, warps per CTA
  Sw16Fn fn;
};

#define ST_CLASS(g, r, c) {g, r, c, kWarps16, sw16_kernel<g, r, c, kWarps16>}
#define ST_CLASS_W(g, r, c, w) {g, r, c, w, sw16_kernel<g, r, c, w>}
static const Sw16Class kClasses[] = {
    ST_CLASS(4, 8, 4),   ST_CLASS(8, 8, 4),   ST_CLASS(16, 8, 4),  ST_CLASS(32, 8, 4),
    ST_CLASS(4, 12, 4),  ST_CLASS(8, 12, 4),  ST_CLASS(16, 12, 4), ST_CLASS(32, 12, 4),
    ST_CLASS(4, 16, 4),  ST_CLASS(8, 16, 4),  ST_CLASS(16, 16, 4), ST_CLASS(32, 16, 4),
    ST_CLASS(4, 20, 4),  ST_CLASS(8, 20, 4),  ST_CLASS(16, 20, 4), ST_CLASS(32, 20, 4),
    ST_CLASS(4, 24, 4),  ST_CLASS(8, 24, 4),  ST_CLASS(16, 24, 4), ST_CLASS(32, 24, 4),
    ST_CLASS_W(4, 28, 4, 4), ST_CLASS_W(8, 28, 4, 4), ST_CLASS_W(16, 28, 4, 4),
    ST_CLASS_W(4, 32, 4, 4), ST_CLASS_W(8, 32, 4, 4), ST_CLASS_W(16, 32, 4, 4),
    ST_CLASS(32, 16, 2),
};
#undef ST_CLASS
#undef ST_CLASS_W
constexpr int kNumClasses = sizeof(kClasses) / sizeof(kClasses[0]);
static_assert(kNumClasses <= kMaxTileClasses, "tile classes exceed the tuning arrays");

int st_tuning_num_classes() { return kNumClasses; }
void st_tuning_class_shape(int c, int* G, int* R, int* C) {
  *G = kClasses[c].G;
  *R = kClasses[c].R;
  *C = kClasses[c].C;
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct ProfileBlock {
  DevMem mem;
  uint32_t live = 0;
};

struct ProfileMeta {
  uint32_t m = 0;
  int32_t max_score = 0;
  bool fits8 = false;
  bool live = false;
  int block = -1;
  const int8_t* p8 = nullptr;
  const int32_t* p32 = nullptr;
  uint32_t stride8 = 0, stride32 = 0;
};

// One per-call scoring in flight (st_sw_score): its own stream, pinned block,
// device staging and scratch, so that calls from several host threads run at
// once; the context lock covers only their set-up and launches.
struct CallSlot {
  cudaStream_t s = nullptr;
  cudaEvent_t ev_in = nullptr;    // the context stream's work before the call (profile tables ready)
  cudaEvent_t ev_done = nullptr;  // the call's result is in the pinned block
  uint64_t epoch = 0;             // the context's profile epoch the slot's stream is ordered after
  Pinned pin;
  DevMem stage, scratch;
};

struct st_ctx {
  int device = 0;
  int sms = 0;
  MemTracker mt;
  cudaStream_t own = nullptr;     // the context's stream (also used for graph capture)
  cudaStream_t copy = nullptr;    // host->device uploads that may overlap queued kernels
  cudaStream_t stream = nullptr;  // where work is launched
  cudaStream_t plan_s = nullptr;  // profile builds and the device planner, beside kernels still queued
  cudaEvent_t plan_ev = nullptr;  // the end of a device plan's preparation on plan_s
  std::recursive_mutex mu;
  uint64_t launches = 0;
  // database
  DevMem db_arena, db_off, db_len;
  std::vector<uint32_t> h_db_len;
  std::vector<uint64_t> h_db_off;  // arena offset of each sequence (multiple of 16)
  // the caller's host arena at the last st_db_upload: its address and offsets[0..n_seqs], so that a
  // lane given as a slice of that arena (the reference's Lane) maps back to a sequence
  uintptr_t h_src_base = 0;
  std::vector<uint64_t> h_src_off;
  uint32_t n_seqs = 0;
  uint32_t max_len = 0;  // longest sequence
  uint64_t n_res = 0;
  bool has_db = false;
  cudaEvent_t db_ev = nullptr;  // after the last stream-ordered change of the database tables
  cudaEvent_t trace_base = nullptr;  // with ST_TRACE: the origin of the batches' device timestamps
  bool db_ev_set = false;
  // profiles
  std::vector<ProfileMeta> profs;
  std::vector<std::unique_ptr<ProfileBlock>> blocks;
  DevMem d_p8, d_p32, d_stride8, d_stride32, d_qlen, d_maxs, d_fits8;
  bool prof_dirty = true;
  uint32_t max_m = 0;
  std::vector<uint32_t> free_ids;  // ids of freed profiles, handed out again
  cudaEvent_t prof_ev = nullptr;   // after the last profile build (work using profiles waits on it)
  bool prof_ev_set = false;
  cudaEvent_t copy_ev = nullptr;   // uploads on the copy stream
  Pinned prof_desc;                // build descriptors on their way to the device
  Pinned plan_meta;                // profile lengths and int8 flags for the device planner's first stage
  Pinned prof_stage[2];            // pageable rows staged on their way to the device
  cudaEvent_t prof_stage_ev[2] = {};
  bool prof_stage_used[2] = {};
  static constexpr int kMetaRing = 4;
  Pinned meta_pin[kMetaRing];      // profile tables on their way to the device
  cudaEvent_t meta_ev[kMetaRing] = {};
  bool meta_used[kMetaRing] = {};
  int meta_slot = 0;
  std::vector<int> free_blocks;    // blocks whose profiles are all freed
  // staging for the per-call paths
  Pinned pin;
  DevMem stage;
  DevMem scratch_small;
  // st_sw_score calls in flight: slots handed out under call_mu (not the context lock)
  static constexpr size_t kMaxCallSlots = 32;
  std::mutex call_mu;
  std::shared_mutex call_rw;  // held shared by per-call scorings from their checks to their launches
  uint64_t prof_epoch = 1;    // changes whenever profile layouts or tables are (re)written on the streams
  std::condition_variable call_cv;
  std::vector<std::unique_ptr<CallSlot>> call_slots;
  std::vector<CallSlot*> call_idle;
  Tuning tuning;
  // seed index over the database (st_seed_index_build): offsets of the 20^w codes, postings
  DevMem seed_off, seed_post;
  SeedPat seed_pat{};
  uint64_t seed_n_post = 0;
  bool has_seed_index = false;
  // device arenas of finished work, reused by later work; an arena with an
  // event is reusable once the event has completed (work queued before it done)
  struct PoolEntry {
    DevMem mem;
    cudaEvent_t ready = nullptr;
  };
  std::vector<PoolEntry> pool;
  std::vector<cudaEvent_t> spare_events;
  // pipelined batches: pinned staging ring (one block per plan in flight) and two side streams
  static constexpr int kStageRing = 6;
  Pinned plan_pin[kStageRing];
  cudaEvent_t plan_pin_ev[kStageRing] = {};
  bool plan_pin_used[kStageRing] = {};
  static constexpr int kMaxSide = 4;
  cudaStream_t side[kMaxSide] = {};
  Pinned out_pin;  // scores and kernel tags on their way to pageable caller buffers
  std::vector<std::unique_ptr<Pinned>> pin_free;  // staging blocks of finished batches
  cudaEvent_t side_ev[1 + kMaxSide] = {};  // [0] start of a batch, [1 + i] end of side stream i's work
  // fork streams of a plan's launches: the 16-bit classes run side by side, the 32-bit kernel after them.
  // Set 0 serves the context's own / caller's stream, set 1 + i side stream i.
  struct ForkSet {
    static constexpr int kForks = 15;
    cudaStream_t s[kForks] = {};
    cudaEvent_t ev[kForks + 1] = {};
  };
  ForkSet forks[1 + kMaxSide];
  // host buffers of the planner, kept between plans so their pages stay mapped
  struct PlanScratch {
    std::vector<uint32_t> pq, pt, tlen, byq, list32;
    std::vector<int32_t> pc, pr;
    std::vector<uint8_t> route;
    std::vector<uint64_t> qstart, n32;
    std::vector<uint32_t> hist;  // per-thread query histograms of the grouping
    std::vector<Sw16Slot> slots[32];
    std::vector<Sw16WarpTask> wt[32];
    std::vector<Sw16CtaTask> cta[32];
  } ps;
};

// A device buffer of at least `bytes` from the context's pool (or a new allocation).
static int pool_get(st_ctx* c, size_t bytes, DevMem& out) {
  int best = -1;
  for (size_t i = 0; i < c->pool.size(); ++i) {
    const DevMem& m = c->pool[i].mem;
    if (m.bytes < bytes || m.bytes > 4 * bytes + (64 << 20)) continue;
    if (best >= 0 && m.bytes >= c->pool[best].mem.bytes) continue;
    cudaEvent_t e = c->pool[i].ready;
    if (e && cudaEventQuery(e) != cudaSuccess) {
      cudaGetLastError();  // cudaErrorNotReady: still in use
      continue;
    }
    best = static_cast<int>(i);
  }
  if (best >= 0) {
    out = std::move(c->pool[best].mem);
    if (c->pool[best].ready) c->spare_events.push_back(c->pool[best].ready);
    c->pool.erase(c->pool.begin() + best);
    return ST_OK;
  }
  // new arenas come in a few size classes (2^k times 1, 1.25, 1.5 or 1.75), so that later requests of a
  // similar size find one to reuse instead of allocating (a large cudaMalloc or cudaFree costs milliseconds)
  size_t cls = 1 << 20;
  while (cls < bytes) cls <<= 1;
  size_t q = cls / 8;  // quarter steps between cls / 2 and cls
  size_t want = cls;
  for (size_t k = 5; k <= 8; ++k)
    if (q * k >= bytes) {
      want = q * k;
      break;
    }
  return dev_alloc(&c->mt, out, std::max(want, bytes));
}

static void pool_trim(st_ctx* c) {
  while (c->pool.size() > 96) {  // keep the most recent arenas (freeing one waits for the device)
    if (c->pool.front().ready) c->spare_events.push_back(c->pool.front().ready);
    c->pool.erase(c->pool.begin());
  }
}

// Back to the pool, reusable at once (no queued work uses it).
static void pool_put(st_ctx* c, DevMem&& m) {
  if (!m.p) return;
  c->pool.push_back(st_ctx::PoolEntry{std::move(m), nullptr});
  pool_trim(c);
}

// Back to the pool, reusable once the work queued on `s` so far has finished.
static void pool_put_after(st_ctx* c, DevMem&& m, cudaStream_t s) {
  if (!m.p) return;
  cudaEvent_t e = nullptr;
  if (!c->spare_events.empty()) {
    e = c->spare_events.back();
    c->spare_events.pop_back();
  } else if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    cudaStreamSynchronize(s);  // no event: wait instead
    pool_put(c, std::move(m));
    return;
  }
  cudaEventRecord(e, s);
  c->pool.push_back(st_ctx::PoolEntry{std::move(m), e});
  pool_trim(c);
}

static DeviceDb db_view(st_ctx* c) {
  DeviceDb d;
  d.arena = c->db_arena.as<uint8_t>();
  d.offset = c->db_off.as<uint64_t>();
  d.length = c->db_len.as<uint32_t>();
  d.n_seqs = c->n_seqs;
  return d;
}

// The context's side stream for short preparatory work (profile layout builds,
// the device planner) that need not queue behind the kernels already on the
// context's stream; at the highest priority, so its kernels take SMs as the
// running grids retire.
static int side_stream(st_ctx* c, cudaStream_t* out) {
  if (!c->plan_s) {
    int lo = 0, hi = 0;
    ST_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    ST_CUDA(cudaStreamCreateWithPriority(&c->plan_s, cudaStreamNonBlocking, hi));
  }
  if (!c->plan_ev) ST_CUDA(cudaEventCreateWithFlags(&c->plan_ev, cudaEventDisableTiming));
  *out = c->plan_s;
  return ST_OK;
}

// Orders the context's stream after the last profile build and, when
// profiles were created or freed since, refreshes the device tables of
// profile pointers, strides and lengths. The tables go up on the stream from
// a ring of pinned blocks, so work already queued keeps reading the old ones.
// Waits for every per-call scoring in flight (before memory they may read is reallocated).
static int calls_drain(st_ctx* c) {
  std::lock_guard<std::mutex> lk(c->call_mu);
  for (auto& sl : c->call_slots)
    if (sl->s) ST_CUDA(cudaStreamSynchronize(sl->s));
  return ST_OK;
}

static CallSlot* call_acquire(st_ctx* c) {
  std::unique_lock<std::mutex> lk(c->call_mu);
  for (;;) {
    if (!c->call_idle.empty()) {
      CallSlot* sl = c->call_idle.back();
      c->call_idle.pop_back();
      return sl;
    }
    if (c->call_slots.size() < st_ctx::kMaxCallSlots) {
      c->call_slots.push_back(std::make_unique<CallSlot>());
      return c->call_slots.back().get();
    }
    c->call_cv.wait(lk);  // every slot is in a call; the first to finish hands its slot over
  }
}

static void call_release(st_ctx* c, CallSlot* sl) {
  {
    std::lock_guard<std::mutex> lk(c->call_mu);
    c->call_idle.push_back(sl);
  }
  c->call_cv.notify_one();
}

static int sync_profiles(st_ctx* c) {
  if (c->prof_ev_set) {
    ST_CUDA(cudaStreamWaitEvent(c->stream, c->prof_ev, 0));
    if (c->own != c->stream) ST_CUDA(cudaStreamWaitEvent(c->own, c->prof_ev, 0));
  }
  if (!c->prof_dirty) return ST_OK;
  const size_t n = std::max<size_t>(c->profs.size(), 1);
  const size_t o_p8 = 0, o_p32 = o_p8 + n * 8, o_s8 = o_p32 + n * 8, o_s32 = o_s8 + n * 4, o_ql = o_s32 + n * 4,
               o_mx = o_ql + n * 4, o_f8 = o_mx + n * 4, total = o_f8 + n;
  const int slot = c->meta_slot;
  c->meta_slot = (slot + 1) % st_ctx::kMetaRing;
  if (!c->meta_ev[slot]) ST_CUDA(cudaEventCreateWithFlags(&c->meta_ev[slot], cudaEventDisableTiming));
  if (c->meta_used[slot]) ST_CUDA(cudaEventSynchronize(c->meta_ev[slot]));  // its last upload is done
  c->meta_used[slot] = false;
  ST_TRY(c->meta_pin[slot].reserve(total));
  char* h = c->meta_pin[slot].as<char>();
  memset(h, 0, total);
  const int8_t** p8 = reinterpret_cast<const int8_t**>(h + o_p8);
  const int32_t** p32 = reinterpret_cast<const int32_t**>(h + o_p32);
  uint32_t* s8 = reinterpret_cast<uint32_t*>(h + o_s8);
  uint32_t* s32 = reinterpret_cast<uint32_t*>(h + o_s32);
  uint32_t* ql = reinterpret_cast<uint32_t*>(h + o_ql);
  int32_t* mx = reinterpret_cast<int32_t*>(h + o_mx);
  uint8_t* f8 = reinterpret_cast<uint8_t*>(h + o_f8);
  uint32_t max_m = 0;
  for (size_t i = 0; i < c->profs.size(); ++i) {
    const ProfileMeta& p = c->profs[i];
    if (!p.live) continue;
    p8[i] = p.p8;
    p32[i] = p.p32;
    s8[i] = p.stride8;
    s32[i] = p.stride32;
    ql[i] = p.m;
    mx[i] = p.max_score;
    f8[i] = p.fits8 ? 1 : 0;
    max_m = std::max(max_m, p.m);
  }
  auto up = [&](DevMem& d, size_t off, size_t bytes) -> int {
    if (d.bytes < bytes) {
      ST_CUDA(cudaStreamSynchronize(c->stream));  // queued work may read the old table
      // and so may per-call scorings: none is between its checks and its launches (they hold the call
      // lock shared), and those launched are waited for
      std::unique_lock<std::shared_mutex> calls(c->call_rw);
      ST_TRY(calls_drain(c));
      ST_TRY(dev_alloc(&c->mt, d, bytes * 2));
    }
    ST_CUDA(cudaMemcpyAsync(d.p, h + off, bytes, cudaMemcpyHostToDevice, c->stream));
    return ST_OK;
  };
  ST_TRY(up(c->d_p8, o_p8, n * 8));
  ST_TRY(up(c->d_p32, o_p32, n * 8));
  ST_TRY(up(c->d_stride8, o_s8, n * 4));
  ST_TRY(up(c->d_stride32, o_s32, n * 4));
  ST_TRY(up(c->d_qlen, o_ql, n * 4));
  ST_TRY(up(c->d_maxs, o_mx, n * 4));
  ST_TRY(up(c->d_fits8, o_f8, n));
  ST_CUDA(cudaEventRecord(c->meta_ev[slot], c->stream));
  if (c->own != c->stream) ST_CUDA(cudaStreamWaitEvent(c->own, c->meta_ev[slot], 0));  // graphs run there too
  c->meta_used[slot] = true;
  c->max_m = max_m;
  c->prof_dirty = false;
  ++c->prof_epoch;
  return ST_OK;
}

static DeviceProfiles prof_view(st_ctx* c) {
  DeviceProfiles p;
  p.p8 = c->d_p8.as<const int8_t* const>();
  p.p32 = c->d_p32.as<const int32_t* const>();
  p.stride8 = c->d_stride8.as<uint32_t>();
  p.stride32 = c->d_stride32.as<uint32_t>();
  p.qlen = c->d_qlen.as<uint32_t>();
  p.max_score = c->d_maxs.as<int32_t>();
  p.fits8 = c->d_fits8.as<uint8_t>();
  return p;
}

static int g_class_smem[kNumClasses];  // dynamic shared memory each 16-bit class may use
static int g_ung_smem = 0;              // dynamic shared memory the ungapped kernels may use
static int g_ung_split_smem = 0;        // the same for ungapped_hits_split_kernel (more static shared memory)
static int g_gate_smem = 0;             // dynamic shared memory of the prefilter segment kernel

static int set_smem_limits(int device) {
  int optin = 0;
  ST_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  for (int i = 0; i < kNumClasses; ++i) {
    cudaFuncAttributes fa;
    ST_CUDA(cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(kClasses[i].fn)));
    g_class_smem[i] = std::min<int>(kMaxSmem, optin - static_cast<int>(fa.sharedSizeBytes));
    ST_CUDA(cudaFuncSetAttribute(kClasses[i].fn, cudaFuncAttributeMaxDynamicSharedMemorySize, g_class_smem[i]));
  }
  cudaFuncAttributes fa_t, fa_f;
  ST_CUDA(cudaFuncGetAttributes(&fa_t, reinterpret_cast<const void*>(ungapped_kernel<true>)));
  ST_CUDA(cudaFuncGetAttributes(&fa_f, reinterpret_cast<const void*>(ungapped_kernel<false>)));
  g_ung_smem = std::min<int>(kMaxSmem, optin - static_cast<int>(std::max(fa_t.sharedSizeBytes, fa_f.sharedSizeBytes)));
  ST_CUDA(cudaFuncSetAttribute(ungapped_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, g_ung_smem));
  ST_CUDA(cudaFuncSetAttribute(ungapped_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, g_ung_smem));
  cudaFuncAttributes fa_r;
  ST_CUDA(cudaFuncGetAttributes(&fa_r, reinterpret_cast<const void*>(ungapped_hits_refill_kernel)));
  g_ung_smem = std::min<int>(g_ung_smem, optin - static_cast<int>(fa_r.sharedSizeBytes));
  ST_CUDA(cudaFuncSetAttribute(ungapped_hits_refill_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, g_ung_smem));
  cudaFuncAttributes fa_s;
  ST_CUDA(cudaFuncGetAttributes(&fa_s, reinterpret_cast<const void*>(ungapped_hits_split_kernel)));
  g_ung_split_smem = std::min<int>(kMaxSmem, optin - static_cast<int>(fa_s.sharedSizeBytes));
  ST_CUDA(cudaFuncSetAttribute(ungapped_hits_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               g_ung_split_smem));
  cudaFuncAttributes fa_g;
  ST_CUDA(cudaFuncGetAttributes(&fa_g, reinterpret_cast<const void*>(gate_score_kernel)));
  g_gate_smem = std::min<int>(kMaxSmem, optin - static_cast<int>(fa_g.sharedSizeBytes));
  ST_CUDA(cudaFuncSetAttribute(gate_score_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, g_gate_smem));
  return ST_OK;
}

extern "C" st_ctx* st_init(int device, size_t hbm_budget_bytes) {
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    fail(ST_ECUDA, "no CUDA device available: %s", cudaGetErrorString(e));
    return nullptr;
  }
  if (device < 0 || device >= ndev) {
    fail(ST_EINVAL, "device %d out of range (have %d)", device, ndev);
    return nullptr;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    fail(ST_ECUDA, "cudaSetDevice(%d) failed", device);
    return nullptr;
  }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  if (prop.major < 10) {
    fail(ST_ECUDA, "device %d is sm_%d%d; this library is built for sm_100a (B200)", device, prop.major,
         prop.minor);
    return nullptr;
  }
  if (!prop.unifiedAddressing) {  // per-call scorings write their results straight into pinned host memory
    fail(ST_ECUDA, "device %d lacks unified addressing", device);
    return nullptr;
  }
  auto c = std::make_unique<st_ctx>();
  c->device = device;
  c->sms = prop.multiProcessorCount;
  c->mt.budget = hbm_budget_bytes;
  if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) {
    fail(ST_ECUDA, "cudaStreamCreate failed");
    return nullptr;
  }
  c->stream = c->own;
  if (cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking) != cudaSuccess) {
    fail(ST_ECUDA, "cudaStreamCreate failed");
    return nullptr;
  }
  if (set_smem_limits(device) != ST_OK) return nullptr;
  tuning_defaults(&c->tuning);
  return c.release();
}

extern "C" void st_shutdown(st_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaStreamSynchronize(c->own);
  for (auto s : c->side)
    if (s) cudaStreamSynchronize(s);
  for (auto s : c->side)
    if (s) cudaStreamDestroy(s);
  for (auto e : c->side_ev)
    if (e) cudaEventDestroy(e);
  for (auto e : c->plan_pin_ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : c->pool)
    if (e.ready) cudaEventDestroy(e.ready);
  for (auto e : c->spare_events) cudaEventDestroy(e);
  for (auto& f : c->forks) {
    for (auto s : f.s)
      if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
    for (auto e : f.ev)
      if (e) cudaEventDestroy(e);
  }
  for (auto& sl : c->call_slots) {
    if (sl->s) {
      cudaStreamSynchronize(sl->s);
      cudaStreamDestroy(sl->s);
    }
    if (sl->ev_in) cudaEventDestroy(sl->ev_in);
    if (sl->ev_done) cudaEventDestroy(sl->ev_done);
  }
  c->call_slots.clear();
  c->call_idle.clear();
  cudaStream_t own = c->own;
  if (c->copy) {
    cudaStreamSynchronize(c->copy);
    cudaStreamDestroy(c->copy);
  }
  if (c->plan_s) {
    cudaStreamSynchronize(c->plan_s);
    cudaStreamDestroy(c->plan_s);
  }
  if (c->db_ev) cudaEventDestroy(c->db_ev);
  if (c->plan_ev) cudaEventDestroy(c->plan_ev);
  if (c->trace_base) cudaEventDestroy(c->trace_base);
  if (c->prof_ev) cudaEventDestroy(c->prof_ev);
  if (c->copy_ev) cudaEventDestroy(c->copy_ev);
  for (auto e : c->meta_ev)
    if (e) cudaEventDestroy(e);
  for (auto e : c->prof_stage_ev)
    if (e) cudaEventDestroy(e);
  delete c;
  cudaStreamDestroy(own);
}

#define CTX_GUARD(c)                                               \
  if (!(c)) return fail(ST_EINVAL, "null context");                \
  std::lock_guard<std::recursive_mutex> lk_((c)->mu);              \
  do {                                                             \
    if (cudaSetDevice((c)->device) != cudaSuccess)                 \
      return fail(ST_ECUDA, "cudaSetDevice(%d) failed", (c)->device); \
  } while (0)

extern "C" int st_set_stream(st_ctx* c, void* s) {
  CTX_GUARD(c);
  c->stream = s ? static_cast<cudaStream_t>(s) : c->own;
  return ST_OK;
}

extern "C" int st_synchronize(st_ctx* c) {
  CTX_GUARD(c);
  ST_CUDA(cudaStreamSynchronize(c->stream));
  ST_CUDA(cudaStreamSynchronize(c->own));
  return ST_OK;
}

extern "C" int st_mem_used(st_ctx* c, uint64_t* bytes) {
  CTX_GUARD(c);
  if (!bytes) return fail(ST_EINVAL, "null output");
  *bytes = c->mt.used;
  return ST_OK;
}

extern "C" int st_launch_count(st_ctx* c, uint64_t* launches) {
  CTX_GUARD(c);
  if (!launches) return fail(ST_EINVAL, "null output");
  *launches = c->launches;
  return ST_OK;
}

// ---------------------------------------------------------------------------
// database
// ---------------------------------------------------------------------------
extern "C" int st_db_upload(st_ctx* c, const uint8_t* residues, const uint64_t* offsets, uint32_t n_seqs) {
  CTX_GUARD(c);
  if (!offsets || (!residues && n_seqs && offsets[n_seqs] > offsets[0]))
    return fail(ST_EINVAL, "st_db_upload: null input");
  std::vector<uint64_t> off(n_seqs + 1);
  std::vector<uint32_t> len(n_seqs);
  uint64_t total = 0;
  for (uint32_t s = 0; s < n_seqs; ++s) {
    if (offsets[s + 1] < offsets[s]) return fail(ST_EINVAL, "st_db_upload: offsets decrease at %u", s);
    const uint64_t l = offsets[s + 1] - offsets[s];
    if (l >= (1ull << 31)) return fail(ST_EINVAL, "st_db_upload: sequence %u longer than 2^31", s);
    off[s] = total;
    len[s] = static_cast<uint32_t>(l);
    total += up16(l);
  }
  off[n_seqs] = total;
  const size_t arena_bytes = total + 32;
  ST_TRY(c->pin.reserve(arena_bytes));
  uint8_t* h = c->pin.as<uint8_t>();
  memset(h, kSentinel, arena_bytes);
  for (uint32_t s = 0; s < n_seqs; ++s) {
    const uint8_t* src = residues + offsets[s];
    uint8_t* dst = h + off[s];
    for (uint32_t i = 0; i < len[s]; ++i) dst[i] = src[i] < kSentinel ? src[i] : kSentinel;
  }
  ST_CUDA(cudaStreamSynchronize(c->stream));
  ST_TRY(dev_alloc(&c->mt, c->db_arena, arena_bytes));
  ST_TRY(dev_alloc(&c->mt, c->db_off, (n_seqs + 1) * sizeof(uint64_t)));
  ST_TRY(dev_alloc(&c->mt, c->db_len, std::max<size_t>(n_seqs, 1) * sizeof(uint32_t)));
  ST_CUDA(cudaMemcpyAsync(c->db_arena.p, h, arena_bytes, cudaMemcpyHostToDevice, c->own));
  ST_CUDA(cudaMemcpyAsync(c->db_off.p, off.data(), off.size() * 8, cudaMemcpyHostToDevice, c->own));
  if (n_seqs) ST_CUDA(cudaMemcpyAsync(c->db_len.p, len.data(), len.size() * 4, cudaMemcpyHostToDevice, c->own));
  ST_CUDA(cudaStreamSynchronize(c->own));
  c->max_len = len.empty() ? 0 : *std::max_element(len.begin(), len.end());
  c->h_db_len = std::move(len);
  c->h_db_off.assign(off.begin(), off.end() - 1);
  c->h_src_base = reinterpret_cast<uintptr_t>(residues);
  c->h_src_off.assign(offsets, offsets + n_seqs + 1);
  c->n_seqs = n_seqs;
  c->n_res = offsets[n_seqs] - offsets[0];
  c->has_db = true;
  c->has_seed_index = false;  // an index describes the previous database
  return ST_OK;
}

extern "C" int st_db_info(st_ctx* c, uint32_t* n_seqs, uint64_t* n_residues) {
  CTX_GUARD(c);
  if (n_seqs) *n_seqs = c->n_seqs;
  if (n_residues) *n_residues = c->n_res;
  return ST_OK;
}

// ---------------------------------------------------------------------------
// profiles
// ---------------------------------------------------------------------------
// Builds the residue-major int8 and int32 layouts of many profiles from their
// [m][21] rows, uploaded as int8 when every score of the profile fits int8 and
// as int32 otherwise: one CTA per profile.
struct ProfBuildDesc {
  uint64_t src;      // first row value: a byte offset into the int8 rows, or an element offset into the int32 rows
  uint64_t o8, o32;  // byte offsets of the int8 / int32 layouts in the block
  uint32_t m, stride8, stride32, fits8;
};

__global__ void __launch_bounds__(256) build_profiles_kernel(const int8_t* __restrict__ rows8,
                                                             const int32_t* __restrict__ rows32,
                                                             const ProfBuildDesc* __restrict__ desc, char* base) {
  const ProfBuildDesc d = desc[blockIdx.x];
  int32_t* p32 = reinterpret_cast<int32_t*>(base + d.o32);
  int8_t* p8 = reinterpret_cast<int8_t*>(base + d.o8);
  const uint32_t total = kProfRows * d.stride32;
  for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const uint32_t r = idx / d.stride32;
    const uint32_t i = idx - r * d.stride32;
    int32_t v = 0;
    if (i < d.m && r < static_cast<uint32_t>(kAlpha)) {
      const size_t at = d.src + static_cast<size_t>(i) * kAlpha + r;
      v = d.fits8 ? static_cast<int32_t>(rows8[at]) : rows32[at];
    }
    p32[idx] = v;
    if (i < d.stride8) p8[static_cast<size_t>(r) * d.stride8 + i] = d.fits8 ? static_cast<int8_t>(v) : 0;
  }
}

extern "C" int st_profiles_create(st_ctx* c, const int32_t* rows, const uint64_t* row_offsets, uint32_t n_profiles,
                                  uint32_t* ids) {
  CTX_GUARD(c);
  if (!row_offsets || !ids || (!rows && n_profiles && row_offsets[n_profiles] > row_offsets[0]))
    return fail(ST_EINVAL, "st_profiles_create: null input");
  if (n_profiles == 0) return ST_OK;
  TraceClock tc("profiles");
  std::vector<ProfBuildDesc> desc(n_profiles);
  std::vector<int32_t> mx(n_profiles);
  for (uint32_t k = 0; k < n_profiles; ++k) {
    if (row_offsets[k + 1] < row_offsets[k]) return fail(ST_EINVAL, "st_profiles_create: offsets decrease");
    if (row_offsets[k + 1] - row_offsets[k] > (1u << 20))
      return fail(ST_EINVAL, "st_profiles_create: query of %llu rows exceeds 2^20",
                  static_cast<unsigned long long>(row_offsets[k + 1] - row_offsets[k]));
  }
  // layouts depend on the lengths only
  size_t bytes8 = 0, bytes32 = 0;
  for (uint32_t k = 0; k < n_profiles; ++k) {
    ProfBuildDesc& x = desc[k];
    x.m = static_cast<uint32_t>(row_offsets[k + 1] - row_offsets[k]);
    x.src = (row_offsets[k] - row_offsets[0]) * kAlpha;  // the profile's int8 slot (moved below if it is int32)
    x.stride8 = static_cast<uint32_t>(std::max<size_t>(up16(x.m), 16));
    x.stride32 = static_cast<uint32_t>(std::max<size_t>(up256(x.m), kSw32Rows));
    x.o32 = bytes32;
    bytes32 += static_cast<size_t>(kProfRows) * x.stride32 * 4;
  }
  for (uint32_t k = 0; k < n_profiles; ++k) {
    desc[k].o8 = bytes32 + bytes8;
    bytes8 += up16(static_cast<size_t>(kProfRows) * desc[k].stride8);
  }
  const size_t rows_total = row_offsets[n_profiles] - row_offsets[0];
  const size_t bytes_r8 = up16(rows_total * kAlpha);  // an int8 slot for every profile's rows
  const size_t desc_bytes = up16(n_profiles * sizeof(ProfBuildDesc));
  // the layouts are built on the side stream, beside kernels already queued on the
  // context's stream; work that reads profiles waits for prof_ev (sync_profiles)
  cudaStream_t bs = nullptr;
  ST_TRY(side_stream(c, &bs));
  // tmp: int8 rows and descriptors; tmp32: int32 rows of the profiles outside int8; both back to the pool
  // once the layouts are built
  DevMem blk_mem, tmp, tmp32;
  ST_TRY(pool_get(c, bytes32 + bytes8, blk_mem));
  ST_TRY(pool_get(c, bytes_r8 + desc_bytes + 16, tmp));
  struct Back {
    st_ctx* c;
    DevMem* m;
    cudaStream_t s;
    ~Back() { pool_put_after(c, std::move(*m), s); }
  } back_tmp{c, &tmp, bs}, back_tmp32{c, &tmp32, bs};
  if (!c->copy_ev) ST_CUDA(cudaEventCreateWithFlags(&c->copy_ev, cudaEventDisableTiming));
  if (!c->prof_ev) ST_CUDA(cudaEventCreateWithFlags(&c->prof_ev, cudaEventDisableTiming));
  tc.lap("alloc");
  char* base = blk_mem.as<char>();
  int8_t* d_r8 = tmp.as<int8_t>();
  ProfBuildDesc* d_desc = reinterpret_cast<ProfBuildDesc*>(tmp.as<char>() + bytes_r8);
  // Host data goes up through the two pinned staging blocks in turn, each uploaded on the copy stream
  // (beside any kernels still queued) while the next one fills; the build runs on the side stream after the
  // uploads.  The call returns once everything is on the device (the caller may reuse the rows), not when
  // the build is done: later work on the profiles is ordered after it.
  constexpr size_t kChunk = 32ull << 20;
  int slot = 0;
  auto stage_slot = [&](size_t bytes, char** h) -> int {
    Pinned& st = c->prof_stage[slot];
    if (!c->prof_stage_ev[slot]) ST_CUDA(cudaEventCreateWithFlags(&c->prof_stage_ev[slot], cudaEventDisableTiming));
    if (c->prof_stage_used[slot]) ST_CUDA(cudaEventSynchronize(c->prof_stage_ev[slot]));
    ST_TRY(st.reserve(std::max(bytes, kChunk)));
    *h = st.as<char>();
    return ST_OK;
  };
  auto stage_send = [&](void* dst, size_t bytes) -> int {
    ST_CUDA(cudaMemcpyAsync(dst, c->prof_stage[slot].p, bytes, cudaMemcpyHostToDevice, c->copy));
    ST_CUDA(cudaEventRecord(c->prof_stage_ev[slot], c->copy));
    c->prof_stage_used[slot] = true;
    slot ^= 1;
    return ST_OK;
  };
  // 1. every profile's rows as int8 (a quarter of the bytes), its score range found in the same pass:
  // residues >= 21 score 0, so the range starts at 0; a profile with a score outside int8 leaves its slot
  // unused and goes up as int32 below
  uint32_t k0 = 0;
  while (k0 < n_profiles) {
    uint32_t k1 = k0 + 1;
    while (k1 < n_profiles && (row_offsets[k1 + 1] - row_offsets[k0]) * kAlpha <= kChunk) ++k1;
    const size_t bytes = (row_offsets[k1] - row_offsets[k0]) * kAlpha;
    char* h = nullptr;
    ST_TRY(stage_slot(bytes, &h));
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t k = k0; k < static_cast<int64_t>(k1); ++k) {
      const size_t cnt = static_cast<size_t>(desc[k].m) * kAlpha;
      const int32_t* r = rows + row_offsets[k] * kAlpha;
      int8_t* d8 = reinterpret_cast<int8_t*>(h) + (row_offsets[k] - row_offsets[k0]) * kAlpha;
      int32_t lo = 0, hi = 0;
      for (size_t i = 0; i < cnt; ++i) {
        const int32_t v = r[i];
        d8[i] = static_cast<int8_t>(v);
        lo = std::min(lo, v);
        hi = std::max(hi, v);
      }
      mx[k] = hi;
      desc[k].fits8 = (lo >= -128 && hi <= 127) ? 1u : 0u;
    }
    if (bytes) ST_TRY(stage_send(d_r8 + (row_offsets[k0] - row_offsets[0]) * kAlpha, bytes));
    k0 = k1;
  }
  // 2. the profiles outside int8, as int32
  std::vector<uint32_t> wide;
  size_t wide_rows = 0;
  for (uint32_t k = 0; k < n_profiles; ++k)
    if (!desc[k].fits8) {
      desc[k].src = wide_rows * kAlpha;
      wide_rows += desc[k].m;
      wide.push_back(k);
    }
  int32_t* d_r32 = nullptr;
  if (wide_rows) {
    ST_TRY(pool_get(c, wide_rows * kAlpha * 4, tmp32));
    d_r32 = tmp32.as<int32_t>();
    size_t w0 = 0;
    while (w0 < wide.size()) {
      size_t w1 = w0 + 1, bytes = static_cast<size_t>(desc[wide[w0]].m) * kAlpha * 4;
      while (w1 < wide.size() && bytes + static_cast<size_t>(desc[wide[w1]].m) * kAlpha * 4 <= kChunk)
        bytes += static_cast<size_t>(desc[wide[w1++]].m) * kAlpha * 4;
      char* h = nullptr;
      ST_TRY(stage_slot(bytes, &h));
      const uint64_t e0 = desc[wide[w0]].src;
#pragma omp parallel for schedule(dynamic, 4)
      for (int64_t j = static_cast<int64_t>(w0); j < static_cast<int64_t>(w1); ++j) {
        const uint32_t k = wide[j];
        memcpy(reinterpret_cast<int32_t*>(h) + (desc[k].src - e0), rows + row_offsets[k] * kAlpha,
               static_cast<size_t>(desc[k].m) * kAlpha * 4);
      }
      ST_TRY(stage_send(d_r32 + e0, bytes));
      w0 = w1;
    }
  }
  tc.lap("range");
  ST_TRY(c->prof_desc.reserve(n_profiles * sizeof(ProfBuildDesc)));
  memcpy(c->prof_desc.p, desc.data(), n_profiles * sizeof(ProfBuildDesc));
  ST_CUDA(cudaMemcpyAsync(d_desc, c->prof_desc.p, n_profiles * sizeof(ProfBuildDesc), cudaMemcpyHostToDevice, c->copy));
  ST_CUDA(cudaEventRecord(c->copy_ev, c->copy));
  ST_CUDA(cudaStreamWaitEvent(bs, c->copy_ev, 0));
  build_profiles_kernel<<<n_profiles, 256, 0, bs>>>(d_r8, d_r32, d_desc, base);
  ++c->launches;
  ST_CUDA(cudaGetLastError());
  ST_CUDA(cudaEventRecord(c->prof_ev, bs));
  c->prof_ev_set = true;
  ++c->prof_epoch;
  ST_CUDA(cudaEventSynchronize(c->copy_ev));
  tc.lap("upload");
  int bi;
  if (!c->free_blocks.empty()) {
    bi = c->free_blocks.back();
    c->free_blocks.pop_back();
  } else {
    bi = static_cast<int>(c->blocks.size());
    c->blocks.push_back(std::make_unique<ProfileBlock>());
  }
  ProfileBlock* blk = c->blocks[bi].get();
  blk->mem = std::move(blk_mem);
  blk->live = n_profiles;
  // freed ids first (in increasing order), then new ones
  if (c->free_ids.size() > 1) std::sort(c->free_ids.begin(), c->free_ids.end(), std::greater<uint32_t>());
  for (uint32_t k = 0; k < n_profiles; ++k) {
    const ProfBuildDesc& x = desc[k];
    ProfileMeta pm;
    pm.m = x.m;
    pm.max_score = mx[k];
    pm.fits8 = x.fits8 != 0;
    pm.live = true;
    pm.block = bi;
    pm.p32 = reinterpret_cast<const int32_t*>(base + x.o32);
    pm.p8 = reinterpret_cast<const int8_t*>(base + x.o8);
    pm.stride8 = x.stride8;
    pm.stride32 = x.stride32;
    if (!c->free_ids.empty()) {
      ids[k] = c->free_ids.back();
      c->free_ids.pop_back();
      c->profs[ids[k]] = pm;
    } else {
      ids[k] = static_cast<uint32_t>(c->profs.size());
      c->profs.push_back(pm);
    }
  }
  c->prof_dirty = true;
  return ST_OK;
}

extern "C" int st_profile_create(st_ctx* c, const int32_t* rows, uint32_t m, uint32_t* id) {
  const uint64_t off[2] = {0, m};
  return st_profiles_create(c, rows, off, 1, id);
}

// Releases one profile; its id is handed out again by a later create. The
// block's device memory goes back to the context's pool when its last
// profile is freed (after work already queued on the stream has finished).
static int profile_free(st_ctx* c, uint32_t id) {
  if (id >= c->profs.size() || !c->profs[id].live) return fail(ST_EINVAL, "unknown profile id %u", id);
  ProfileMeta& p = c->profs[id];
  p.live = false;
  ProfileBlock* b = c->blocks[p.block].get();
  if (--b->live == 0) {
    // reusable once work queued so far is done, the block's layout build included
    if (c->prof_ev_set && cudaStreamWaitEvent(c->stream, c->prof_ev, 0) != cudaSuccess)
      return fail(ST_ECUDA, "cudaStreamWaitEvent failed");
    pool_put_after(c, std::move(b->mem), c->stream);
    c->free_blocks.push_back(p.block);
  }
  p.block = -1;
  c->free_ids.push_back(id);
  c->prof_dirty = true;
  return ST_OK;
}

extern "C" int st_profile_free(st_ctx* c, uint32_t id) {
  CTX_GUARD(c);
  return profile_free(c, id);
}

extern "C" int st_profiles_free(st_ctx* c, const uint32_t* ids, uint32_t n) {
  CTX_GUARD(c);
  if (n && !ids) return fail(ST_EINVAL, "st_profiles_free: null ids");
  for (uint32_t k = 0; k < n; ++k) ST_TRY(profile_free(c, ids[k]));
  return ST_OK;
}

static int check_profile(st_ctx* c, uint32_t id) {
  if (id >= c->profs.size() || !c->profs[id].live) return fail(ST_EINVAL, "unknown profile id %u", id);
  return ST_OK;
}

// ---------------------------------------------------------------------------
// planning
// ---------------------------------------------------------------------------
static inline bool gaps16_ok(int32_t open, int32_t ext) {
  // E, F >= -open-ext and H - open >= -open must stay inside int16
  return open >= 0 && ext >= 0 && static_cast<int64_t>(open) + ext <= 16384;
}

static int64_t linear_pos_sum(int64_t s, int64_t e, int64_t a, int b) {
  // sum over i in [s, e] of max(0, a + b*i), b in {-1, 0, 1}
  if (e < s) return 0;
  if (b == 0) return a > 0 ? (e - s + 1) * a : 0;
  if (b == 1) {
    const int64_t i0 = std::max(s, 1 - a);
    if (i0 > e) return 0;
    const int64_t k = e - i0 + 1;
    return k * a + (i0 + e) * k / 2;
  }
  const int64_t i1 = std::min(e, a - 1);
  if (i1 < s) return 0;
  const int64_t k = i1 - s + 1;
  return k * a - (s + i1) * k / 2;
}

static uint64_t band_cells(uint32_t m, uint32_t n, int64_t c, int64_t r) {
  // cells (i, j), 1-based, with |j - i - c| <= r: row i spans [max(1, i+c-r), min(n, i+c+r)]
  if (m == 0 || n == 0 || r < 0) return 0;
  int64_t p1 = 2 - c + r;                   // from here on the left end is i + c - r
  int64_t p2 = static_cast<int64_t>(n) - c - r + 1;  // from here on the right end is n
  const int64_t lo = 1, hi = static_cast<int64_t>(m) + 1;
  p1 = std::min(std::max(p1, lo), hi);
  p2 = std::min(std::max(p2, lo), hi);
  const int64_t cuts[4] = {lo, std::min(p1, p2), std::max(p1, p2), hi};
  int64_t total = 0;
  for (int g = 0; g < 3; ++g) {
    const int64_t s = cuts[g], e = cuts[g + 1] - 1;
    if (e < s) continue;
    const bool left1 = s + c - r <= 1;
    const bool rightA = s + c + r <= static_cast<int64_t>(n);
    int64_t a;
    int b;
    if (left1 && rightA) {
      a = c + r;
      b = 1;
    } else if (left1) {
      a = n;
      b = 0;
    } else if (rightA) {
      a = 2 * r + 1;
      b = 0;
    } else {
      a = static_cast<int64_t>(n) - c + r + 1;
      b = -1;
    }
    total += linear_pos_sum(s, e, a, b);
  }
  return static_cast<uint64_t>(total);
}

struct ClassPlan {
  int cls = -1;
  std::vector<Sw16CtaTask> cta;
  std::vector<Sw16WarpTask> wt;
  std::vector<Sw16Slot> slots;
  size_t o_cta = 0, o_wt = 0, o_slots = 0, o_scratch = 0;  // offsets in the plan's device arena
  uint32_t grid = 0;
  uint32_t smem = 0;
  uint32_t scratch_stride = 0;
  uint64_t cells = 0;     // sum of m*n over this class's pairs
  uint64_t streamed = 0;  // cells the wavefront streams (padded rows x padded columns x slots)
  Sw16Params prm;
};

struct st_plan {
  st_ctx* ctx = nullptr;
  uint64_t n = 0;
  int32_t open = 0, ext = 0;
  int32_t* d_scores = nullptr;
  uint32_t* d_kernels = nullptr;
  std::vector<ClassPlan> classes;
  DevMem arena;  // every device buffer of the plan (from the context's pool)
  uint32_t* counters = nullptr;
  const uint32_t* counters_init = nullptr;
  uint32_t n_static32 = 0;
  uint32_t grid32 = 0, scratch32_stride = 0;
  uint64_t cells = 0;
  uint64_t cells32 = 0;  // cells of pairs sent to the 32-bit kernel at plan time (band cells for bands)
  uint64_t streamed = 0;  // cells streamed by the 16-bit classes
  uint32_t kernels_per_run = 0;
  Sw32Params p32;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

static int occupancy_grid(st_ctx* c, const void* fn, int threads, size_t smem, uint32_t work, uint32_t* grid);

// Grid of the 32-bit kernel: two CTAs per SM for the rare rescores the 16-bit
// classes flag at run time; for a long static list (banded pairs, wide rows,
// gap costs outside 16 bits) as many as the SMs hold; never more warps than
// the run has pairs (a one-pair batch would otherwise carry pass scratch lines
// for 2 x 148 CTAs); bounded so the pass scratch stays within 1 GiB.
static int grid_sw32(st_ctx* c, uint64_t n_static, uint64_t n_pairs, uint32_t scratch_stride, uint32_t* grid) {
  const uint64_t want = std::min<uint64_t>(std::max<uint64_t>(2ull * c->sms, (n_static + kWarps32 - 1) / kWarps32),
                                           std::max<uint64_t>(1, (n_pairs + kWarps32 - 1) / kWarps32));
  ST_TRY(occupancy_grid(c, reinterpret_cast<const void*>(sw32_kernel<kWarps32>), kWarps32 * 32, 0,
                        static_cast<uint32_t>(std::min<uint64_t>(want, 1u << 20)), grid));
  if (scratch_stride) {
    const uint64_t cap = (1ull << 30) / (static_cast<uint64_t>(kWarps32) * scratch_stride * sizeof(int2));
    *grid = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(*grid, cap)));
  }
  return ST_OK;
}

static int occupancy_grid(st_ctx* c, const void* fn, int threads, size_t smem, uint32_t work, uint32_t* grid) {
  int nb = 0;
  ST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem));
  if (nb < 1) return fail(ST_EINVAL, "kernel does not fit on an SM (smem %zu)", smem);
  *grid = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(static_cast<uint64_t>(nb) * c->sms, work)));
  return ST_OK;
}

// The launches of one run, in stream order: clear outputs, reset counters,
// every 16-bit class, then the 32-bit kernel over the static list plus the
// pairs the 16-bit classes flagged.
// With a fork set, the largest class runs on `st` and the others on fork
// streams (forked and joined through events, which graph capture records as
// parallel branches), so the tail of one class overlaps the others.
static int plan_enqueue(st_plan* p, cudaStream_t st, st_ctx::ForkSet* fs, bool graph = false) {
  if (p->n) {
    if (cudaMemsetAsync(p->d_scores, 0, p->n * 4, st) != cudaSuccess) return ST_ECUDA;
    if (p->d_kernels && cudaMemsetAsync(p->d_kernels, 0, p->n * 4, st) != cudaSuccess) return ST_ECUDA;
  }
  if (cudaMemcpyAsync(p->counters, p->counters_init, (kNumClasses + 2) * 4, cudaMemcpyDeviceToDevice, st) !=
      cudaSuccess)
    return ST_ECUDA;
  const size_t nc = p->classes.size();
  const bool band16 = p->p32.band16 != 0;
  if (!fs || nc + (band16 ? 1 : 0) <= 1) {
    for (auto& cp : p->classes) kClasses[cp.cls].fn<<<cp.grid, kClasses[cp.cls].W * 32, cp.smem, st>>>(cp.prm);
    if (band16) sw16_band_kernel<kWarps32><<<p->grid32, kWarps32 * 32, 0, st>>>(p->p32);
  } else {
    // The classes run side by side: the costliest on the launching stream, the
    // others on forks joined before sw32. The launch order matters, as the block
    // scheduler serves the grids in that order:
    // * direct launches: the costliest first, the others by decreasing cost, so
    //   the grids run longest first and the small classes fill the tails of the
    //   large ones (21.3 ms for the 1.2 M-pair PSSM batch, against 22.3 ms with
    //   the costliest launched last);
    // * captured into a graph, whose launch order of independent nodes is the
    //   runtime's: the forks in class order, the costliest last, measured fastest
    //   there (21.1 ms, against 21.7 ms with the costliest captured first).
    // Launch priorities by cost were tried: they also order one batch's classes,
    // but a batch queued behind a running one then jumps ahead of its small
    // classes and delays its completion.
    size_t order[kNumClasses];
    for (size_t i = 0; i < nc; ++i) order[i] = i;
    size_t big = 0;
    for (size_t i = 1; i < nc; ++i)
      if (p->classes[i].cells > p->classes[big].cells) big = i;
    if (graph) {
      std::stable_partition(order, order + nc, [&](size_t i) { return i != big; });
    } else {
      std::stable_sort(order, order + nc,
                       [&](size_t a, size_t b) { return p->classes[a].cells > p->classes[b].cells; });
      big = order[0];
    }
    if (cudaEventRecord(fs->ev[0], st) != cudaSuccess) return ST_ECUDA;
    bool used[st_ctx::ForkSet::kForks] = {};
    int next = 0;
    for (size_t r = 0; r < nc; ++r) {
      const ClassPlan& cp = p->classes[order[r]];
      cudaStream_t s = st;
      if (order[r] != big) {
        const int j = next++ % st_ctx::ForkSet::kForks;
        if (!used[j] && cudaStreamWaitEvent(fs->s[j], fs->ev[0], 0) != cudaSuccess) return ST_ECUDA;
        used[j] = true;
        s = fs->s[j];
      }
      kClasses[cp.cls].fn<<<cp.grid, kClasses[cp.cls].W * 32, cp.smem, s>>>(cp.prm);
      if (cudaGetLastError() != cudaSuccess) return ST_ECUDA;
    }
    if (band16) {  // the banded pairs of the static list, beside the classes (it reads only that list)
      cudaStream_t s = st;
      if (nc > 0) {
        const int j = next++ % st_ctx::ForkSet::kForks;
        if (!used[j] && cudaStreamWaitEvent(fs->s[j], fs->ev[0], 0) != cudaSuccess) return ST_ECUDA;
        used[j] = true;
        s = fs->s[j];
      }
      sw16_band_kernel<kWarps32><<<p->grid32, kWarps32 * 32, 0, s>>>(p->p32);
      if (cudaGetLastError() != cudaSuccess) return ST_ECUDA;
    }
    for (int j = 0; j < st_ctx::ForkSet::kForks; ++j) {
      if (!used[j]) continue;
      if (cudaEventRecord(fs->ev[1 + j], fs->s[j]) != cudaSuccess) return ST_ECUDA;
      if (cudaStreamWaitEvent(st, fs->ev[1 + j], 0) != cudaSuccess) return ST_ECUDA;
    }
  }
  // the band kernel used the 32-bit kernel's work counter
  if (band16 && cudaMemsetAsync(p->p32.work_counter, 0, 4, st) != cudaSuccess) return ST_ECUDA;
  sw32_kernel<kWarps32><<<p->grid32, kWarps32 * 32, 0, st>>>(p->p32);
  return cudaGetLastError() == cudaSuccess ? ST_OK : ST_ECUDA;
}

static int fork_set(st_ctx* c, int i, st_ctx::ForkSet** out) {
  st_ctx::ForkSet& f = c->forks[i];
  for (auto& s : f.s)
    if (!s) ST_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  for (auto& e : f.ev)
    if (!e) ST_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  *out = &f;
  return ST_OK;
}

// Builds a plan for `n` pairs. Its initialised data is staged in pinned block
// `slot` of the context's ring and uploaded on `up`; the block is reused only
// after that copy has finished (an event per block).
static int plan_build(st_ctx* c, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext, int32_t* d_scores,
                      uint32_t* d_kernels, st_plan** out, bool capture, cudaStream_t up, int slot) {
  if (!c->has_db) return fail(ST_ESTATE, "no target database uploaded (st_db_upload)");
  if (n > 0xFFFFFFF0ull) return fail(ST_EINVAL, "too many pairs (%llu)", static_cast<unsigned long long>(n));
  ST_TRY(sync_profiles(c));
  auto plan = std::make_unique<st_plan>();
  plan->ctx = c;
  plan->n = n;
  plan->open = open;
  plan->ext = ext;
  plan->d_scores = d_scores;
  plan->d_kernels = d_kernels;
  const bool g16 = gaps16_ok(open, ext);
  // the longest query whose int8 profile fits the shared memory of some 16-bit class;
  // longer ones take the 32-bit kernel
  uint32_t max_m16 = 0;
  for (int k = 0; k < kNumClasses; ++k) {
    const uint32_t rows = static_cast<uint32_t>(kClasses[k].G * kClasses[k].R);
    const uint32_t smem = static_cast<uint32_t>(std::min<int>(g_class_smem[k], 216 * 1024));  // the models' limit
    max_m16 = std::max(max_m16, smem / kProfRows / rows * rows);
  }
  TraceClock tc("plan");

  auto& ps = c->ps;
  std::vector<uint32_t>& pq = ps.pq;
  std::vector<uint32_t>& pt = ps.pt;
  std::vector<uint32_t>& tlen = ps.tlen;
  std::vector<int32_t>& pc = ps.pc;
  std::vector<int32_t>& pr = ps.pr;
  std::vector<uint8_t>& route = ps.route;  // 0: score 0 (empty), 1: 16-bit kernel, 2: 32-bit kernel
  pq.resize(n);
  pt.resize(n);
  tlen.resize(n);
  pc.resize(n);
  pr.resize(n);
  route.resize(n);
  const uint32_t n_prof = static_cast<uint32_t>(c->profs.size());
  int64_t bad = -1;
  uint64_t cells = 0, cells32 = 0;
  uint32_t max_len = 0, max_m32 = 0;
  // classify every pair (validation, route, cells), in parallel
#pragma omp parallel for schedule(static) reduction(+ : cells, cells32) reduction(max : max_len, max_m32)
  for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
    const st_pair& p = pairs[i];
    if (p.profile >= n_prof || !c->profs[p.profile].live || p.target >= c->n_seqs) {
#pragma omp critical
      if (bad < 0 || i < bad) bad = i;
      continue;
    }
    pq[i] = p.profile;
    pt[i] = p.target;
    pc[i] = p.band_center;
    pr[i] = p.band_radius;
    const ProfileMeta& pm = c->profs[p.profile];
    const uint32_t tl = c->h_db_len[p.target];
    tlen[i] = tl;
    if (pm.m == 0 || tl == 0) {
      route[i] = 0;
      continue;
    }
    max_len = std::max(max_len, tl);
    max_m32 = std::max(max_m32, pm.m);  // every 16-bit pair may be rescored in 32 bits
    if (p.band_radius >= 0) {
      const uint64_t bc = band_cells(pm.m, tl, p.band_center, p.band_radius);
      cells += bc;
      cells32 += bc;
      route[i] = 2;
    } else {
      const uint64_t mc = static_cast<uint64_t>(pm.m) * tl;
      cells += mc;
      if (g16 && pm.fits8 && pm.m <= max_m16) {
        route[i] = 1;
      } else {
        route[i] = 2;
        cells32 += mc;
      }
    }
  }
  if (bad >= 0) {
    const st_pair& p = pairs[bad];
    if (p.profile >= n_prof || !c->profs[p.profile].live)
      return fail(ST_EINVAL, "pair %lld: unknown profile id %u", static_cast<long long>(bad), p.profile);
    return fail(ST_EINVAL, "pair %lld: target %u outside the database (%u sequences)", static_cast<long long>(bad),
                p.target, c->n_seqs);
  }
  plan->cells = cells;
  plan->cells32 = cells32;
  tc.lap("classify");
  // 32-bit list in pair order; 16-bit pairs grouped by query, in pair order
  // within a query: a counting sort with one histogram per thread over
  // contiguous ranges of pairs, so the result is the serial one.
  std::vector<uint32_t>& list32 = ps.list32;
  std::vector<uint64_t>& qstart = ps.qstart;
  qstart.assign(static_cast<size_t>(n_prof) + 1, 0);
  const int nt = std::max(1, std::min(omp_get_max_threads(), static_cast<int>((n + 32767) / 32768)));
  ps.hist.assign(static_cast<size_t>(nt) * n_prof, 0);
  ps.n32.assign(static_cast<size_t>(nt) + 1, 0);
#pragma omp parallel num_threads(nt)
  {
    const int t = omp_get_thread_num();
    const uint64_t i0 = n * t / nt, i1 = n * (t + 1) / nt;
    uint32_t* h = ps.hist.data() + static_cast<size_t>(t) * n_prof;
    uint64_t k32 = 0;
    for (uint64_t i = i0; i < i1; ++i) {
      if (route[i] == 1) ++h[pq[i]];
      else if (route[i] == 2) ++k32;
    }
    ps.n32[t + 1] = k32;
  }
  // per query: start of the query, then each thread's start inside it
  for (uint32_t q = 0; q < n_prof; ++q) {
    uint64_t sum = 0;
    for (int t = 0; t < nt; ++t) sum += ps.hist[static_cast<size_t>(t) * n_prof + q];
    qstart[q + 1] = qstart[q] + sum;
  }
  for (int t = 0; t < nt; ++t) ps.n32[t + 1] += ps.n32[t];
  list32.resize(ps.n32[nt]);
  std::vector<uint32_t>& byq = ps.byq;
  byq.resize(qstart[n_prof]);
#pragma omp parallel for schedule(static)
  for (int64_t q = 0; q < static_cast<int64_t>(n_prof); ++q) {
    uint64_t o = qstart[q];
    for (int t = 0; t < nt; ++t) {
      uint32_t& h = ps.hist[static_cast<size_t>(t) * n_prof + q];
      const uint32_t cnt = h;
      h = static_cast<uint32_t>(o - qstart[q]);  // becomes the thread's offset inside the query
      o += cnt;
    }
  }
#pragma omp parallel num_threads(nt)
  {
    const int t = omp_get_thread_num();
    const uint64_t i0 = n * t / nt, i1 = n * (t + 1) / nt;
    uint32_t* h = ps.hist.data() + static_cast<size_t>(t) * n_prof;
    uint64_t k32 = ps.n32[t];
    for (uint64_t i = i0; i < i1; ++i) {
      if (route[i] == 1) byq[qstart[pq[i]] + h[pq[i]]++] = static_cast<uint32_t>(i);
      else if (route[i] == 2) list32[k32++] = static_cast<uint32_t>(i);
    }
  }
  // The 32-bit list longest first (its kernels pull entries in order), by the steps a warp spends on a pair:
  // passes x (streamed columns + ramp), a banded pair streaming one 256-row pass's band window per pass.
  // The packed band kernel scores neighbouring entries together, so similar pairs share a warp.
  if (list32.size() > 1) {
    std::vector<std::pair<uint64_t, uint32_t>> ord(list32.size());
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < static_cast<int64_t>(list32.size()); ++k) {
      const uint32_t i = list32[k];
      const uint64_t m = c->profs[pq[i]].m, tl = tlen[i];
      const uint64_t P = (m + kSw32Rows - 1) / kSw32Rows;
      uint64_t w = tl;
      if (pr[i] >= 0) w = std::min<uint64_t>(tl, static_cast<uint64_t>(kSw32Rows) + 2 * static_cast<uint64_t>(pr[i]));
      ord[k] = {P * (w + 31), i};
    }
    std::stable_sort(ord.begin(), ord.end(), [](const std::pair<uint64_t, uint32_t>& a,
                                                 const std::pair<uint64_t, uint32_t>& b) { return a.first > b.first; });
    for (size_t k = 0; k < ord.size(); ++k) list32[k] = ord[k].second;
  }
  tc.lap("group");
  // per query (in parallel): targets longest first, then the tile class
  std::vector<uint32_t> qlist;
  for (uint32_t q = 0; q < n_prof; ++q)
    if (qstart[q + 1] > qstart[q]) qlist.push_back(q);
  std::vector<int> qclass(qlist.size());
  std::vector<uint64_t> qsum(qlist.size());
  int toolong = -1;
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t k = 0; k < static_cast<int64_t>(qlist.size()); ++k) {
    const uint32_t q = qlist[k];
    uint32_t* v0 = byq.data() + qstart[q];
    uint32_t* v1 = byq.data() + qstart[q + 1];
    std::stable_sort(v0, v1, [&](uint32_t a, uint32_t b) { return tlen[a] > tlen[b]; });
    thread_local std::vector<uint32_t> tl_desc;
    tl_desc.resize(v1 - v0);
    uint64_t sum_n = 0;
    for (uint32_t* it = v0; it != v1; ++it) {
      tl_desc[it - v0] = tlen[*it];
      sum_n += tlen[*it];
    }
    const uint32_t m = c->profs[q].m;
    const uint32_t mean_n = static_cast<uint32_t>(sum_n / (v1 - v0));
    int cls = tuning_pick_batch(&c->tuning, m, tl_desc.data(), tl_desc.size(), mean_n);
    if (cls < 0) cls = tuning_pick_single(&c->tuning, m, mean_n);  // no class has a rate: the wavefront model
    const uint32_t rows = kClasses[cls].G * kClasses[cls].R;
    const uint32_t P = (m + rows - 1) / rows;
    if (static_cast<uint64_t>(kProfRows) * P * rows > static_cast<uint64_t>(g_class_smem[cls])) {
#pragma omp critical
      toolong = static_cast<int>(m);
    }
    qclass[k] = cls;
    qsum[k] = sum_n;
  }
  if (toolong >= 0) return fail(ST_EINVAL, "query of %d rows does not fit the shared-memory profile", toolong);
  tc.lap("sort+pick");
  std::vector<ClassPlan> cps(kNumClasses);
  for (int k = 0; k < kNumClasses; ++k) {
    cps[k].cls = k;
    cps[k].slots.swap(ps.slots[k]);  // borrow the kept buffers (returned below)
    cps[k].wt.swap(ps.wt[k]);
    cps[k].cta.swap(ps.cta[k]);
  }
  // Emission. A query's pairs (sorted by target length, longest first) form
  // warp tasks of S = 64/G pairs; consecutive warp tasks form CTA tasks. A CTA
  // task ends at 128 warp tasks, or (once it holds a warp task for each warp)
  // when its estimated cost would pass the class's cap: one CTA's share of the
  // class's total cost on a grid of two CTAs per SM. The cap keeps a long
  // query from becoming one CTA task longer than the rest of the launch (the
  // tail); a looser split would pay the ramp, drain and barrier wait of a CTA
  // task more often.
  // Passes: warp-task counts and costs, CTA-task counts, offsets, parallel fill.
  struct QEmit {
    uint32_t n_wt, n_cta;
    size_t wt_off, slot_off, cta_off;
    uint64_t cost, streamed;
  };
  std::vector<QEmit> qe(qlist.size());
  constexpr uint32_t kMaxWtPerCta = 128;

  struct QShape {
    uint32_t S, P, rows, min_cols, step_cost, C;
  };
  auto shape_of = [&](int64_t k) {
    const Sw16Class& kc = kClasses[qclass[k]];
    QShape sh;
    sh.S = 64 / kc.G;
    sh.rows = static_cast<uint32_t>(kc.G * kc.R);
    sh.P = std::max<uint32_t>(1, (c->profs[qlist[k]].m + sh.rows - 1) / sh.rows);
    sh.min_cols = sh.P > 1 ? static_cast<uint32_t>(up16(std::max(32, kc.C * kc.G))) : 32u;
    sh.step_cost = static_cast<uint32_t>(kc.R * kc.C + 8);
    sh.C = static_cast<uint32_t>(kc.C);
    return sh;
  };
  // columns of warp task w of query k: its first pair has the longest target
  auto wt_cols = [&](int64_t k, const QShape& sh, uint32_t w) {
    const uint32_t* v = byq.data() + qstart[qlist[k]];
    return std::max<uint32_t>(sh.min_cols, static_cast<uint32_t>(up4(tlen[v[static_cast<size_t>(w) * sh.S]])));
  };
  auto wt_cost = [&](const QShape& sh, uint32_t ncols) {
    return static_cast<uint64_t>(sh.P) * (ncols / sh.C) * sh.step_cost;
  };
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t k = 0; k < static_cast<int64_t>(qlist.size()); ++k) {
    const QShape sh = shape_of(k);
    const uint64_t np = qstart[qlist[k] + 1] - qstart[qlist[k]];
    QEmit& e = qe[k];
    e.n_wt = static_cast<uint32_t>((np + sh.S - 1) / sh.S);
    e.cost = 0;
    e.streamed = 0;
    for (uint32_t w = 0; w < e.n_wt; ++w) {
      const uint32_t nc = wt_cols(k, sh, w);
      e.cost += wt_cost(sh, nc);
      e.streamed += static_cast<uint64_t>(sh.P) * sh.rows * nc * sh.S;
    }
  }
  std::vector<uint64_t> cap(kNumClasses, 0);
  for (size_t k = 0; k < qlist.size(); ++k) cap[qclass[k]] += qe[k].cost;
  for (int k = 0; k < kNumClasses; ++k) cap[k] = std::max<uint64_t>(1, cap[k] / (2 * c->sms));
  // calls f(w0, w1, cost) for each CTA task of query k, in order
  auto for_each_cta = [&](int64_t k, const QShape& sh, auto&& f) {
    const uint32_t n_wt = qe[k].n_wt;
    const uint64_t cp = cap[qclass[k]];
    uint32_t w0 = 0;
    uint64_t acc = 0;
    for (uint32_t w = 0; w < n_wt; ++w) {
      const uint64_t cw = wt_cost(sh, wt_cols(k, sh, w));
      const uint32_t cnt = w - w0;
      if (cnt == kMaxWtPerCta || (cnt >= static_cast<uint32_t>(kClasses[qclass[k]].W) && acc + cw > cp)) {
        f(w0, w, acc);
        w0 = w;
        acc = 0;
      }
      acc += cw;
    }
    if (n_wt > w0) f(w0, n_wt, acc);
  };
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t k = 0; k < static_cast<int64_t>(qlist.size()); ++k) {
    uint32_t n = 0;
    for_each_cta(k, shape_of(k), [&](uint32_t, uint32_t, uint64_t) { ++n; });
    qe[k].n_cta = n;
  }
  std::vector<size_t> n_wt_cls(kNumClasses, 0), n_slot_cls(kNumClasses, 0), n_cta_cls(kNumClasses, 0);
  for (size_t k = 0; k < qlist.size(); ++k) {
    const uint32_t q = qlist[k];
    const int cls = qclass[k];
    const uint32_t S = 64 / kClasses[cls].G;
    QEmit& e = qe[k];
    e.wt_off = n_wt_cls[cls];
    e.slot_off = n_slot_cls[cls];
    e.cta_off = n_cta_cls[cls];
    n_wt_cls[cls] += e.n_wt;
    n_slot_cls[cls] += static_cast<size_t>(e.n_wt) * S;
    n_cta_cls[cls] += e.n_cta;
    cps[cls].cells += static_cast<uint64_t>(c->profs[q].m) * qsum[k];
    cps[cls].streamed += e.streamed;
    plan->streamed += e.streamed;
  }
  std::vector<std::vector<uint64_t>> cta_cost(kNumClasses);
  for (int k = 0; k < kNumClasses; ++k) {
    cps[k].wt.resize(n_wt_cls[k]);
    cps[k].slots.resize(n_slot_cls[k]);
    cps[k].cta.resize(n_cta_cls[k]);
    cta_cost[k].resize(n_cta_cls[k]);
  }
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t k = 0; k < static_cast<int64_t>(qlist.size()); ++k) {
    const uint32_t q = qlist[k];
    const int cls = qclass[k];
    ClassPlan& cp = cps[cls];
    const QEmit& e = qe[k];
    const QShape sh = shape_of(k);
    const uint32_t* v = byq.data() + qstart[q];
    const size_t np = qstart[q + 1] - qstart[q];
    for (uint32_t w = 0; w < e.n_wt; ++w) {
      const size_t sb = e.slot_off + static_cast<size_t>(w) * sh.S;
      uint32_t ncols = sh.min_cols;
      for (uint32_t sidx = 0; sidx < sh.S; ++sidx) {
        const size_t j = static_cast<size_t>(w) * sh.S + sidx;
        Sw16Slot sl{kNoPair, 0, 0, 0};
        if (j < np) {
          const uint32_t pi = v[j];
          sl.pair = pi;
          sl.toff16 = static_cast<uint32_t>(c->h_db_off[pt[pi]] / 16);
          sl.tlen16 = static_cast<uint32_t>(up16(tlen[pi]));
          sl.tlen = tlen[pi];
          ncols = std::max<uint32_t>(ncols, static_cast<uint32_t>(up4(tlen[pi])));
        }
        cp.slots[sb + sidx] = sl;
      }
      cp.wt[e.wt_off + w] = Sw16WarpTask{static_cast<uint32_t>(sb), ncols};
    }
    size_t t = e.cta_off;
    for_each_cta(k, sh, [&](uint32_t w0, uint32_t w1, uint64_t cost) {
      cp.cta[t] = Sw16CtaTask{q, static_cast<uint32_t>(e.wt_off + w0), static_cast<uint32_t>(e.wt_off + w1),
                              sh.P * sh.rows};
      cta_cost[cls][t] = cost;
      ++t;
    });
  }
  tc.lap("emit");
  // order CTA tasks by estimated cost, longest first
  for (auto& cp : cps) {
    if (cp.cta.empty()) continue;
    const auto& cost0 = cta_cost[cp.cls];
    std::vector<uint32_t> idx(cp.cta.size());
    std::iota(idx.begin(), idx.end(), 0u);
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return cost0[a] > cost0[b]; });
    std::vector<Sw16CtaTask> sorted(cp.cta.size());
    for (size_t i = 0; i < idx.size(); ++i) sorted[i] = cp.cta[idx[i]];
    cp.cta.swap(sorted);
  }

  tc.lap("lpt");
  // launch shapes and scratch needs
  uint32_t nonempty = 0;
  for (auto& cp : cps) {
    if (cp.cta.empty()) continue;
    ++nonempty;
    const Sw16Class& k = kClasses[cp.cls];
    uint32_t max_mpad = 0, max_cols = 0;
    bool multi = false;
    for (auto& t : cp.cta) {
      max_mpad = std::max(max_mpad, t.m_pad);
      if (t.m_pad > static_cast<uint32_t>(k.G * k.R)) multi = true;
    }
    for (auto& w : cp.wt) max_cols = std::max(max_cols, w.ncols);
    cp.smem = kProfRows * max_mpad;
    ST_TRY(occupancy_grid(c, reinterpret_cast<const void*>(k.fn), k.W * 32, cp.smem,
                          static_cast<uint32_t>(cp.cta.size()), &cp.grid));
    cp.scratch_stride = multi ? max_cols : 0;
  }
  plan->scratch32_stride = max_m32 > static_cast<uint32_t>(kSw32Rows) ? max_len : 0;
  plan->n_static32 = static_cast<uint32_t>(list32.size());
  ST_TRY(grid_sw32(c, plan->n_static32, n, plan->scratch32_stride, &plan->grid32));

  // one device arena: [initialised data (one upload)] [scratch]
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    const size_t o = off;
    off = (off + bytes + 255) & ~static_cast<size_t>(255);
    return o;
  };
  const size_t o_pq = carve(n * 4), o_pt = carve(n * 4), o_pc = carve(n * 4), o_pr = carve(n * 4);
  const size_t o_list = carve(std::max<uint64_t>(n, 1) * 4);
  const size_t o_cinit = carve((kNumClasses + 2) * 4);
  for (auto& cp : cps) {
    if (cp.cta.empty()) continue;
    cp.o_cta = carve(cp.cta.size() * sizeof(Sw16CtaTask));
    cp.o_wt = carve(cp.wt.size() * sizeof(Sw16WarpTask));
    cp.o_slots = carve(cp.slots.size() * sizeof(Sw16Slot));
  }
  uint32_t zcols = 64;
  for (auto& cp : cps)
    for (auto& w : cp.wt) zcols = std::max(zcols, w.ncols + 8);
  const size_t o_zline = carve(static_cast<size_t>(zcols) * sizeof(uint2));
  const size_t data_bytes = off;
  const size_t o_cnt = carve((kNumClasses + 2) * 4);
  for (auto& cp : cps) {
    if (cp.cta.empty() || !cp.scratch_stride) continue;
    const size_t groups = static_cast<size_t>(cp.grid) * kClasses[cp.cls].W * (32 / kClasses[cp.cls].G);
    cp.o_scratch = carve(groups * cp.scratch_stride * sizeof(uint2));
  }
  const size_t o_s32 = carve(plan->scratch32_stride
                                 ? static_cast<size_t>(plan->grid32) * kWarps32 * plan->scratch32_stride * sizeof(int2)
                                 : 16);
  const size_t total_bytes = off;
  tc.lap("shapes");
  if (trace_on())
    for (auto& cp : cps)
      if (!cp.cta.empty())
        fprintf(stderr, "[st] plan class %d: %zu CTA tasks, %zu warp tasks, grid %u, smem %u, scratch %u\n", cp.cls,
                cp.cta.size(), cp.wt.size(), cp.grid, cp.smem, cp.scratch_stride);
  ST_TRY(pool_get(c, total_bytes, plan->arena));
  tc.lap("arena");
  char* dbase = plan->arena.as<char>();
  // stage the data region in pinned memory and upload it at once
  Pinned& pin = c->plan_pin[slot];
  if (!c->plan_pin_ev[slot]) ST_CUDA(cudaEventCreateWithFlags(&c->plan_pin_ev[slot], cudaEventDisableTiming));
  if (c->plan_pin_used[slot]) ST_CUDA(cudaEventSynchronize(c->plan_pin_ev[slot]));  // may still feed a copy
  c->plan_pin_used[slot] = false;
  ST_TRY(pin.reserve(data_bytes));
  char* h = pin.as<char>();
#pragma omp parallel sections
  {
#pragma omp section
    memcpy(h + o_pq, pq.data(), n * 4);
#pragma omp section
    memcpy(h + o_pt, pt.data(), n * 4);
#pragma omp section
    memcpy(h + o_pc, pc.data(), n * 4);
#pragma omp section
    memcpy(h + o_pr, pr.data(), n * 4);
  }
  if (!list32.empty()) memcpy(h + o_list, list32.data(), list32.size() * 4);
  {
    // input of a first pass: H = 0 above the query, F = first-row F
    uint2* z = reinterpret_cast<uint2*>(h + o_zline);
    const uint2 v = make_uint2(0u, pk_splat(-open));
    for (uint32_t i = 0; i < zcols; ++i) z[i] = v;
  }
  {
    // counters: [0, kNumClasses) class work, [kNumClasses] 32-bit work, [kNumClasses+1] list count
    uint32_t* ci = reinterpret_cast<uint32_t*>(h + o_cinit);
    for (int k = 0; k < kNumClasses + 2; ++k) ci[k] = 0;
    ci[kNumClasses + 1] = plan->n_static32;
  }
  for (auto& cp : cps) {
    if (cp.cta.empty()) continue;
    memcpy(h + cp.o_cta, cp.cta.data(), cp.cta.size() * sizeof(Sw16CtaTask));
    memcpy(h + cp.o_wt, cp.wt.data(), cp.wt.size() * sizeof(Sw16WarpTask));
    const size_t ns = cp.slots.size();
    const Sw16Slot* src = cp.slots.data();
    Sw16Slot* dst = reinterpret_cast<Sw16Slot*>(h + cp.o_slots);
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < static_cast<int64_t>((ns + 65535) / 65536); ++b) {
      const size_t a0 = static_cast<size_t>(b) * 65536, a1 = std::min(ns, a0 + 65536);
      memcpy(dst + a0, src + a0, (a1 - a0) * sizeof(Sw16Slot));
    }
  }
  ST_CUDA(cudaMemcpyAsync(dbase, h, data_bytes, cudaMemcpyHostToDevice, up));
  ST_CUDA(cudaEventRecord(c->plan_pin_ev[slot], up));
  c->plan_pin_used[slot] = true;
  tc.lap("stage+upload");
  plan->counters = reinterpret_cast<uint32_t*>(dbase + o_cnt);
  plan->counters_init = reinterpret_cast<const uint32_t*>(dbase + o_cinit);
  for (auto& cp : cps) {
    if (!cp.cta.empty()) {
      ClassPlan kept;
      kept.cls = cp.cls;
      kept.cta.assign(cp.cta.begin(), cp.cta.end());  // small: one entry per query and class
      kept.grid = cp.grid;
      kept.smem = cp.smem;
      kept.scratch_stride = cp.scratch_stride;
      kept.cells = cp.cells;
      kept.streamed = cp.streamed;
      kept.o_cta = cp.o_cta;
      kept.o_wt = cp.o_wt;
      kept.o_slots = cp.o_slots;
      kept.o_scratch = cp.o_scratch;
      plan->classes.push_back(std::move(kept));
    }
    ps.slots[cp.cls].swap(cp.slots);
    ps.wt[cp.cls].swap(cp.wt);
    ps.cta[cp.cls].swap(cp.cta);
  }

  const DeviceDb db = db_view(c);
  const DeviceProfiles pv = prof_view(c);
  uint32_t* counters = plan->counters;
  const uint32_t* d_pair_q = reinterpret_cast<const uint32_t*>(dbase + o_pq);
  const uint32_t* d_pair_t = reinterpret_cast<const uint32_t*>(dbase + o_pt);
  const int32_t* d_pair_c = reinterpret_cast<const int32_t*>(dbase + o_pc);
  const int32_t* d_pair_r = reinterpret_cast<const int32_t*>(dbase + o_pr);
  uint32_t* d_list = reinterpret_cast<uint32_t*>(dbase + o_list);

  // kernel parameters (kept on the plan: the graph and the per-class profiler launch the same)
  for (auto& cp : plan->classes) {
    Sw16Params& prm = cp.prm;
    prm.arena = db.arena;
    prm.prof = pv;
    prm.cta_tasks = reinterpret_cast<const Sw16CtaTask*>(dbase + cp.o_cta);
    prm.n_cta_tasks = static_cast<uint32_t>(cp.cta.size());
    prm.warp_tasks = reinterpret_cast<const Sw16WarpTask*>(dbase + cp.o_wt);
    prm.slots = reinterpret_cast<const Sw16Slot*>(dbase + cp.o_slots);
    prm.scores = d_scores;
    prm.kernels = d_kernels;
    prm.ovf_count = counters + kNumClasses + 1;
    prm.ovf_pairs = d_list;
    prm.work_counter = counters + cp.cls;
    prm.scratch = reinterpret_cast<uint2*>(dbase + cp.o_scratch);
    prm.zline = reinterpret_cast<const uint2*>(dbase + o_zline);
    prm.scratch_stride = cp.scratch_stride;
    prm.open = open;
    prm.ext = ext;
  }
  {
    Sw32Params& p32 = plan->p32;
    p32.db = db;
    p32.prof = pv;
    p32.list = d_list;
    p32.list_count = counters + kNumClasses + 1;
    p32.pair_query = d_pair_q;
    p32.pair_target = d_pair_t;
    p32.pair_center = d_pair_c;
    p32.pair_radius = d_pair_r;
    p32.scores = d_scores;
    p32.kernels = d_kernels;
    p32.work_counter = counters + kNumClasses;
    p32.scratch = reinterpret_cast<int2*>(dbase + o_s32);
    p32.scratch_stride = plan->scratch32_stride;
    p32.open = open;
    p32.ext = ext;
    p32.n_static = plan->n_static32;
    p32.band16 = (g16 && plan->n_static32 > 0) ? 1u : 0u;
  }

  plan->kernels_per_run = static_cast<uint32_t>(plan->classes.size()) + 1 + plan->p32.band16;
  if (capture) {
    // capture a run into a CUDA graph on the context's own stream (ordered after the upload)
    ST_CUDA(cudaStreamSynchronize(up));
    ST_CUDA(cudaStreamBeginCapture(c->own, cudaStreamCaptureModeThreadLocal));
    st_ctx::ForkSet* fs = nullptr;
    ST_TRY(fork_set(c, 0, &fs));
    const int rc = plan_enqueue(plan.get(), c->own, fs, true);
    cudaError_t ce = cudaStreamEndCapture(c->own, &plan->graph);
    if (rc != ST_OK || ce != cudaSuccess)
      return fail(ST_ECUDA, "graph capture failed: %s", cudaGetErrorString(ce != cudaSuccess ? ce : cudaGetLastError()));
    ST_CUDA(cudaGraphInstantiate(&plan->exec, plan->graph, 0));
  }
  *out = plan.release();
  return ST_OK;
}

static int plan_run(st_plan* p) {
  st_ctx* c = p->ctx;
  if (p->exec) {
    ST_CUDA(cudaGraphLaunch(p->exec, c->stream));
  } else {
    st_ctx::ForkSet* fs = nullptr;
    ST_TRY(fork_set(c, 0, &fs));
    if (plan_enqueue(p, c->stream, fs) != ST_OK)
      return fail(ST_ECUDA, "plan launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  c->launches += p->kernels_per_run;
  return ST_OK;
}

static void plan_free(st_plan* p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  pool_put(p->ctx, std::move(p->arena));
  delete p;
}

extern "C" int st_plan_create(st_ctx* c, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext,
                              int32_t* d_scores, uint32_t* d_kernels, st_plan** plan) {
  CTX_GUARD(c);
  if (!plan || (n && (!pairs || !d_scores))) return fail(ST_EINVAL, "st_plan_create: null argument");
  return plan_build(c, pairs, n, open, ext, d_scores, d_kernels, plan, true, c->stream, 0);
}

extern "C" int st_plan_run(st_plan* p) {
  if (!p) return fail(ST_EINVAL, "null plan");
  st_ctx* c = p->ctx;
  CTX_GUARD(c);
  return plan_run(p);
}

extern "C" int st_plan_stats(st_plan* p, uint64_t* cells, uint64_t* rescored, uint32_t* n_classes) {
  if (!p) return fail(ST_EINVAL, "null plan");
  st_ctx* c = p->ctx;
  CTX_GUARD(c);
  if (cells) *cells = p->cells;
  if (n_classes) *n_classes = static_cast<uint32_t>(p->classes.size());
  if (rescored) {
    uint32_t cnt = 0;
    ST_CUDA(cudaStreamSynchronize(c->stream));
    ST_CUDA(cudaMemcpy(&cnt, p->counters + kNumClasses + 1, 4, cudaMemcpyDeviceToHost));
    *rescored = cnt >= p->n_static32 ? cnt - p->n_static32 : 0;
  }
  return ST_OK;
}

extern "C" int st_plan_profile(st_plan* p, uint32_t cap, int32_t* classes, uint64_t* cells, float* ms,
                               uint32_t* n_out) {
  if (!p) return fail(ST_EINVAL, "null plan");
  st_ctx* c = p->ctx;
  CTX_GUARD(c);
  if (!n_out || (cap && (!classes || !cells || !ms))) return fail(ST_EINVAL, "st_plan_profile: null output");
  const uint32_t nb = p->p32.band16 ? 1u : 0u;
  const uint32_t n = static_cast<uint32_t>(p->classes.size()) + 1 + nb;
  *n_out = n;
  if (cap < n) return fail(ST_EINVAL, "st_plan_profile: room for %u entries needed", n);
  cudaEvent_t e0, e1;
  ST_CUDA(cudaEventCreate(&e0));
  ST_CUDA(cudaEventCreate(&e1));
  ST_CUDA(cudaMemcpyAsync(p->counters, p->counters_init, (kNumClasses + 2) * 4, cudaMemcpyDeviceToDevice,
                          c->stream));
  for (uint32_t i = 0; i < n; ++i) {
    ST_CUDA(cudaEventRecord(e0, c->stream));
    if (i < p->classes.size()) {
      const ClassPlan& cp = p->classes[i];
      kClasses[cp.cls].fn<<<cp.grid, kClasses[cp.cls].W * 32, cp.smem, c->stream>>>(cp.prm);
      classes[i] = cp.cls;
      cells[i] = cp.cells;
    } else if (nb && i + 1 < n) {
      // the banded pairs of the static list (their cells are counted with the 32-bit list's)
      sw16_band_kernel<kWarps32><<<p->grid32, kWarps32 * 32, 0, c->stream>>>(p->p32);
      ST_CUDA(cudaMemsetAsync(p->p32.work_counter, 0, 4, c->stream));
      classes[i] = -2;
      cells[i] = 0;
    } else {
      // every 16-bit class has run: the list holds the static and the rescored pairs
      sw32_kernel<kWarps32><<<p->grid32, kWarps32 * 32, 0, c->stream>>>(p->p32);
      classes[i] = -1;
      cells[i] = p->cells32;
    }
    ST_CUDA(cudaEventRecord(e1, c->stream));
    ST_CUDA(cudaEventSynchronize(e1));
    ST_CUDA(cudaEventElapsedTime(&ms[i], e0, e1));
    ++c->launches;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ST_OK;
}

extern "C" void st_plan_destroy(st_plan* p) {
  if (!p) return;
  st_ctx* c = p->ctx;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  plan_free(p);
}

// Pipelining of large batches: chunks of about 320K pairs (ST_PIPELINE_PAIRS
// overrides; 0 turns pipelining off), the first two a quarter and a half of
// that so the GPU starts early, rotating over side streams
// (ST_PIPELINE_STREAMS, 1 to 4). Returns the chunk boundaries (one chunk: no
// pipelining).
static std::vector<uint64_t> pipeline_bounds(uint64_t n) {
  const uint64_t chunk = env_u64("ST_PIPELINE_PAIRS", 320 * 1024);
  std::vector<uint64_t> b{0};
  if (chunk == 0 || n < chunk + chunk / 2) {
    b.push_back(n);
    return b;
  }
  const uint64_t first[2] = {std::max<uint64_t>(1, chunk / 4), std::max<uint64_t>(1, chunk / 2)};
  uint64_t at = 0;
  for (int k = 0; k < 2 && n - at > chunk + chunk / 2; ++k) b.push_back(at += first[k]);
  const uint64_t rest = n - at;
  const uint64_t m = std::min<uint64_t>(62, std::max<uint64_t>(1, (rest + chunk / 2) / chunk));
  for (uint64_t k = 1; k <= m; ++k) b.push_back(at + rest * k / m);
  return b;
}

static int pipeline_streams() {
  return static_cast<int>(std::min<uint64_t>(st_ctx::kMaxSide, std::max<uint64_t>(1, env_u64("ST_PIPELINE_STREAMS", 4))));
}

// Checks every pair (profile id live, target in the database) in parallel;
// reports the first bad one. Also the longest target and query of the batch
// (the 32-bit kernel's scratch).
static int validate_pairs(st_ctx* c, const st_pair* pairs, uint64_t n, uint32_t* max_len, uint32_t* max_m) {
  const uint32_t n_prof = static_cast<uint32_t>(c->profs.size());
  int64_t bad = INT64_MAX;
  uint32_t ml = 0, mm = 0;
#pragma omp parallel for schedule(static) reduction(min : bad) reduction(max : ml, mm)
  for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
    const st_pair& p = pairs[i];
    if (p.profile >= n_prof || !c->profs[p.profile].live || p.target >= c->n_seqs) {
      bad = std::min<int64_t>(bad, i);
      continue;
    }
    const uint32_t tl = c->h_db_len[p.target];
    const uint32_t m = c->profs[p.profile].m;
    if (tl && m) {
      ml = std::max(ml, tl);
      mm = std::max(mm, m);
    }
  }
  if (bad != INT64_MAX) {
    const st_pair& p = pairs[bad];
    if (p.profile >= n_prof || !c->profs[p.profile].live)
      return fail(ST_EINVAL, "pair %lld: unknown profile id %u", static_cast<long long>(bad), p.profile);
    return fail(ST_EINVAL, "pair %lld: target %u outside the database (%u sequences)", static_cast<long long>(bad),
                p.target, c->n_seqs);
  }
  if (max_len) *max_len = ml;
  if (max_m) *max_m = mm;
  return ST_OK;
}

static int bits_for(uint64_t x) {
  int b = 0;
  while (x) {
    ++b;
    x >>= 1;
  }
  return std::max(b, 1);
}

// Builds the plan of pairs[0..n) on the device (st_dplan.cuh), on the
// context's stream, with one synchronisation to read the per-class totals
// that size the rest. `work` holds the per-pair and per-query buffers and
// must outlive the plan's runs; the plan owns the task arrays and scratch.
static int upload_host(st_ctx* c, void* dst, const void* src, size_t bytes, cudaStream_t s);

static int dplan_build(st_ctx* c, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext, int32_t* d_scores,
                       uint32_t* d_kernels, uint32_t max_len, uint32_t max_m, DevMem& work, st_plan** out) {
  cudaStream_t st = c->stream;
  TraceClock tc("dplan");
  const uint32_t n_prof = static_cast<uint32_t>(c->profs.size());
  const bool g16 = gaps16_ok(open, ext);
  auto plan = std::make_unique<st_plan>();
  plan->ctx = c;
  plan->n = n;
  plan->open = open;
  plan->ext = ext;
  plan->d_scores = d_scores;
  plan->d_kernels = d_kernels;

  DpClasses cls{};
  cls.n = kNumClasses;
  cls.sms = static_cast<uint32_t>(c->sms);
  uint32_t max_m16 = 0;
  for (int k = 0; k < kNumClasses; ++k) {
    DpClass& d = cls.c[k];
    d.G = kClasses[k].G;
    d.R = kClasses[k].R;
    d.C = kClasses[k].C;
    d.W = kClasses[k].W;
    d.rows = d.G * d.R;
    d.S = 64 / d.G;
    const uint32_t smem = static_cast<uint32_t>(std::min<int>(g_class_smem[k], 216 * 1024));
    d.max_mpad = smem / kProfRows / d.rows * d.rows;
    d.rate = c->tuning.rate[k];
    max_m16 = std::max(max_m16, d.max_mpad);
  }
  memcpy(cls.table, c->tuning.table, sizeof(cls.table));

  DpIn in{};
  in.n = static_cast<uint32_t>(n);
  in.db = db_view(c);
  in.prof = prof_view(c);
  in.n_prof = n_prof;
  in.max_m16 = max_m16;
  in.g16 = g16 ? 1u : 0u;
  in.tbits = static_cast<uint32_t>(bits_for(max_len));
  const int key_bits = std::min(64, bits_for(n_prof) + static_cast<int>(in.tbits));

  // scratch sizes of the library sorts and scans (host-side queries)
  using ull = unsigned long long;
  size_t t_sort = 0, t_qsort = 0, t_scan = 0;
  {
    cub::DoubleBuffer<ull> kb(nullptr, nullptr);
    cub::DoubleBuffer<uint32_t> vb(nullptr, nullptr);
    ST_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t_sort, kb, vb, static_cast<int>(n), 0, key_bits, st));
    cub::DoubleBuffer<uint32_t> qk(nullptr, nullptr), qv(nullptr, nullptr);
    ST_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t_qsort, qk, qv, static_cast<int>(n_prof), 0, 6, st));
    ST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t_scan, static_cast<uint32_t*>(nullptr),
                                          static_cast<uint32_t*>(nullptr), static_cast<int>(n_prof + 1), st));
  }
  const size_t t_tmp = std::max(t_sort, std::max(t_qsort, t_scan));
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    const size_t o = off;
    off = (off + bytes + 255) & ~static_cast<size_t>(255);
    return o;
  };
  const size_t np1 = static_cast<size_t>(n_prof) + 1;
  const size_t o_pairs = carve(n * 16), o_pq = carve(n * 4), o_pt = carve(n * 4), o_pc = carve(n * 4),
               o_pr = carve(n * 4), o_k0 = carve(n * 8), o_k1 = carve(n * 8), o_v0 = carve(n * 4),
               o_v1 = carve(n * 4), o_list = carve(n * 4), o_cnt = carve((kNumClasses + 2) * 4),
               o_cinit = carve((kNumClasses + 2) * 4), o_qcnt = carve(np1 * 4), o_qstart = carve(np1 * 4),
               o_qclass = carve(np1 * 4), o_nwt = carve(np1 * 4), o_ncta = carve(np1 * 4), o_qk0 = carve(np1 * 4),
               o_qk1 = carve(np1 * 4), o_qi0 = carve(np1 * 4), o_qi1 = carve(np1 * 4), o_as = carve(np1 * 4),
               o_aw = carve(np1 * 4), o_ac = carve(np1 * 4), o_os = carve(np1 * 4), o_ow = carve(np1 * 4),
               o_oc = carve(np1 * 4), o_tot = carve(sizeof(DpTotals)), o_sq = carve(np1 * 4),
               o_sf = carve(np1), o_tmp = carve(t_tmp);
  ST_TRY(pool_get(c, off, work));
  char* b = work.as<char>();
  DpWork w{};
  w.pq = reinterpret_cast<uint32_t*>(b + o_pq);
  w.pt = reinterpret_cast<uint32_t*>(b + o_pt);
  w.pc = reinterpret_cast<int32_t*>(b + o_pc);
  w.pr = reinterpret_cast<int32_t*>(b + o_pr);
  w.keys = reinterpret_cast<ull*>(b + o_k0);
  w.keys_alt = reinterpret_cast<ull*>(b + o_k1);
  w.vals = reinterpret_cast<uint32_t*>(b + o_v0);
  w.vals_alt = reinterpret_cast<uint32_t*>(b + o_v1);
  w.list32 = reinterpret_cast<uint32_t*>(b + o_list);
  uint32_t* counters = reinterpret_cast<uint32_t*>(b + o_cnt);
  uint32_t* cinit = reinterpret_cast<uint32_t*>(b + o_cinit);
  w.list_count = cinit + kNumClasses + 1;  // the static 32-bit list count is the runs' initial list count
  w.qcnt = reinterpret_cast<uint32_t*>(b + o_qcnt);
  w.qstart = reinterpret_cast<uint32_t*>(b + o_qstart);
  w.qclass = reinterpret_cast<uint32_t*>(b + o_qclass);
  w.nwt = reinterpret_cast<uint32_t*>(b + o_nwt);
  w.ncta = reinterpret_cast<uint32_t*>(b + o_ncta);
  w.qkey = reinterpret_cast<uint32_t*>(b + o_qk0);
  w.qkey_alt = reinterpret_cast<uint32_t*>(b + o_qk1);
  w.qid = reinterpret_cast<uint32_t*>(b + o_qi0);
  w.qid_alt = reinterpret_cast<uint32_t*>(b + o_qi1);
  w.a_slots = reinterpret_cast<uint32_t*>(b + o_as);
  w.a_wt = reinterpret_cast<uint32_t*>(b + o_aw);
  w.a_cta = reinterpret_cast<uint32_t*>(b + o_ac);
  w.o_slots = reinterpret_cast<uint32_t*>(b + o_os);
  w.o_wt = reinterpret_cast<uint32_t*>(b + o_ow);
  w.o_cta = reinterpret_cast<uint32_t*>(b + o_oc);
  w.totals = reinterpret_cast<DpTotals*>(b + o_tot);
  void* tmp = b + o_tmp;
  in.pairs = reinterpret_cast<const st_pair*>(b + o_pairs);

  // stage 1: pairs in, classify, sort, per-query class and CTA-task counts, class order.
  // It runs on the planner's own stream, so its one wait (for the per-class
  // totals) does not wait for kernels still queued on the stream, e.g. the
  // previous batch. It reads the pairs and a snapshot of the profiles'
  // lengths and int8 flags, both uploaded on the copy stream, and the
  // database lengths (ordered after any stream-ordered database change).
  if (!c->copy_ev) ST_CUDA(cudaEventCreateWithFlags(&c->copy_ev, cudaEventDisableTiming));
  cudaStream_t s1 = nullptr;
  ST_TRY(side_stream(c, &s1));
  ST_TRY(c->plan_meta.reserve(np1 * 5));
  {
    uint32_t* hq = c->plan_meta.as<uint32_t>();
    uint8_t* hf = c->plan_meta.as<uint8_t>(np1 * 4);
    hq[n_prof] = 0;
    hf[n_prof] = 0;
    for (uint32_t k = 0; k < n_prof; ++k) {
      const ProfileMeta& pm = c->profs[k];
      hq[k] = pm.live ? pm.m : 0;
      hf[k] = pm.live && pm.fits8 ? 1 : 0;
    }
  }
  // the pairs: straight from pinned memory, through the pinned staging blocks from pageable memory
  ST_TRY(upload_host(c, b + o_pairs, pairs, n * 16, s1));
  ST_CUDA(cudaMemcpyAsync(b + o_sq, c->plan_meta.p, np1 * 4, cudaMemcpyHostToDevice, c->copy));
  ST_CUDA(cudaMemcpyAsync(b + o_sf, c->plan_meta.as<uint8_t>(np1 * 4), np1, cudaMemcpyHostToDevice, c->copy));
  ST_CUDA(cudaEventRecord(c->copy_ev, c->copy));
  ST_CUDA(cudaStreamWaitEvent(s1, c->copy_ev, 0));
  if (c->db_ev_set) ST_CUDA(cudaStreamWaitEvent(s1, c->db_ev, 0));
  DpIn in1 = in;
  in1.prof.qlen = reinterpret_cast<const uint32_t*>(b + o_sq);
  in1.prof.fits8 = reinterpret_cast<const uint8_t*>(b + o_sf);
  ST_CUDA(cudaMemsetAsync(cinit, 0, (kNumClasses + 2) * 4, s1));
  ST_CUDA(cudaMemsetAsync(w.qcnt, 0, np1 * 4, s1));
  ST_CUDA(cudaMemsetAsync(w.totals, 0, sizeof(DpTotals), s1));
  const uint32_t gb = static_cast<uint32_t>(std::min<uint64_t>((n + 255) / 256, static_cast<uint64_t>(c->sms) * 8));
  dp_classify_kernel<<<gb, 256, 0, s1>>>(in1, w);
  cub::DoubleBuffer<ull> kb(w.keys, w.keys_alt);
  cub::DoubleBuffer<uint32_t> vb(w.vals, w.vals_alt);
  ST_CUDA(cub::DeviceRadixSort::SortPairs(tmp, t_sort, kb, vb, static_cast<int>(n), 0, key_bits, s1));
  w.vals_sorted = vb.Current();
  ST_CUDA(cub::DeviceScan::ExclusiveSum(tmp, t_scan, w.qcnt, w.qstart, static_cast<int>(np1), s1));
  const uint32_t gq32 = static_cast<uint32_t>((static_cast<uint64_t>(n_prof) * 32 + 255) / 256);
  const uint32_t gq = static_cast<uint32_t>((np1 + 255) / 256);
  dp_pick_kernel<<<gq32, 256, 0, s1>>>(in1, w, cls);
  dp_split_kernel<<<gq, 256, 0, s1>>>(in1, w, cls);
  cub::DoubleBuffer<uint32_t> qk(w.qkey, w.qkey_alt), qi(w.qid, w.qid_alt);
  ST_CUDA(cub::DeviceRadixSort::SortPairs(tmp, t_qsort, qk, qi, static_cast<int>(n_prof), 0, 6, s1));
  w.qid_sorted = qi.Current();
  dp_counts_kernel<<<gq, 256, 0, s1>>>(in1, w, cls);
  ST_CUDA(cub::DeviceScan::ExclusiveSum(tmp, t_scan, w.a_slots, w.o_slots, static_cast<int>(np1), s1));
  ST_CUDA(cub::DeviceScan::ExclusiveSum(tmp, t_scan, w.a_wt, w.o_wt, static_cast<int>(np1), s1));
  ST_CUDA(cub::DeviceScan::ExclusiveSum(tmp, t_scan, w.a_cta, w.o_cta, static_cast<int>(np1), s1));
  ST_CUDA(cudaGetLastError());
  c->launches += 5;
  DpTotals tot;
  uint32_t n_list32 = 0;  // pairs the classify stage sent to the 32-bit kernel
  ST_CUDA(cudaMemcpyAsync(&tot, w.totals, sizeof(DpTotals), cudaMemcpyDeviceToHost, s1));
  ST_CUDA(cudaMemcpyAsync(&n_list32, w.list_count, 4, cudaMemcpyDeviceToHost, s1));
  ST_CUDA(cudaStreamSynchronize(s1));
  tc.lap("stage 1 (device)");

  // stage 2: sizes known; task arrays, scratch, emission, LPT order
  uint64_t n_slots = 0, n_wt = 0, n_cta = 0;
  uint64_t cta_begin[kNumClasses];
  uint32_t zcols = 64;
  for (int k = 0; k < kNumClasses; ++k) {
    cta_begin[k] = n_cta;
    n_slots += static_cast<uint64_t>(tot.n_wt[k]) * (64 / kClasses[k].G);
    n_wt += tot.n_wt[k];
    n_cta += tot.n_cta[k];
    if (tot.n_cta[k]) zcols = std::max(zcols, tot.max_cols[k] + 8);
  }
  for (int k = 0; k < kNumClasses; ++k) {
    if (!tot.n_cta[k]) continue;
    ClassPlan cp;
    cp.cls = k;
    cp.cells = tot.cost[k];  // the fork puts the costliest class on the launching stream
    cp.smem = kProfRows * tot.max_mpad[k];
    ST_TRY(occupancy_grid(c, reinterpret_cast<const void*>(kClasses[k].fn), kClasses[k].W * 32, cp.smem,
                          tot.n_cta[k], &cp.grid));
    cp.scratch_stride = tot.max_cols_multi[k];
    plan->classes.push_back(std::move(cp));
  }
  plan->scratch32_stride = max_m > static_cast<uint32_t>(kSw32Rows) ? max_len : 0;
  plan->n_static32 = n_list32;
  ST_TRY(grid_sw32(c, n_list32, n, plan->scratch32_stride, &plan->grid32));
  if (n_list32 > 1) {
    // the 32-bit list longest first (the packed band kernel scores neighbouring entries together), in the
    // stage-1 buffers that are free now: both key buffers and the value buffer the pair sort left unused
    uint32_t* vfree = w.vals_sorted == w.vals ? w.vals_alt : w.vals;
    size_t t_ls = 0;
    {
      cub::DoubleBuffer<ull> lk(nullptr, nullptr);
      cub::DoubleBuffer<uint32_t> lv(nullptr, nullptr);
      ST_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t_ls, lk, lv, static_cast<int>(n_list32), 0, 48, s1));
    }
    if (t_ls <= t_tmp) {
      const uint32_t gl = static_cast<uint32_t>(std::min<uint64_t>((n_list32 + 255) / 256,
                                                                   static_cast<uint64_t>(c->sms) * 8));
      dp_list_keys_kernel<<<gl, 256, 0, s1>>>(in, w, n_list32, w.keys, vfree);
      cub::DoubleBuffer<ull> lk(w.keys, w.keys_alt);
      cub::DoubleBuffer<uint32_t> lv(vfree, w.list32);
      ST_CUDA(cub::DeviceRadixSort::SortPairs(tmp, t_ls, lk, lv, static_cast<int>(n_list32), 0, 48, s1));
      if (lv.Current() != w.list32)
        ST_CUDA(cudaMemcpyAsync(w.list32, lv.Current(), static_cast<size_t>(n_list32) * 4, cudaMemcpyDeviceToDevice,
                                s1));
    }
  }
  size_t t_lpt = 0;
  {
    cub::DoubleBuffer<ull> ck(nullptr, nullptr);
    cub::DoubleBuffer<uint32_t> ci(nullptr, nullptr);
    ST_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t_lpt, ck, ci, static_cast<int>(n_cta), 0, 44 + 6, st));
  }
  off = 0;
  const size_t p_slots = carve(n_slots * sizeof(Sw16Slot)), p_wt = carve(n_wt * sizeof(Sw16WarpTask)),
               p_craw = carve(n_cta * sizeof(Sw16CtaTask)), p_cta = carve(n_cta * sizeof(Sw16CtaTask)),
               p_ck0 = carve(n_cta * 8), p_ck1 = carve(n_cta * 8), p_ci0 = carve(n_cta * 4),
               p_ci1 = carve(n_cta * 4), p_z = carve(static_cast<size_t>(zcols) * sizeof(uint2)),
               p_tmp = carve(t_lpt);
  for (auto& cp : plan->classes) {
    if (!cp.scratch_stride) continue;
    const size_t groups = static_cast<size_t>(cp.grid) * kClasses[cp.cls].W * (32 / kClasses[cp.cls].G);
    cp.o_scratch = carve(groups * cp.scratch_stride * sizeof(uint2));
  }
  const size_t p_s32 = carve(plan->scratch32_stride ? static_cast<size_t>(plan->grid32) * kWarps32 *
                                                          plan->scratch32_stride * sizeof(int2)
                                                    : 16);
  ST_TRY(pool_get(c, off, plan->arena));
  char* a = plan->arena.as<char>();
  DpOut o{};
  o.slots = reinterpret_cast<Sw16Slot*>(a + p_slots);
  o.wt = reinterpret_cast<Sw16WarpTask*>(a + p_wt);
  o.cta_raw = reinterpret_cast<Sw16CtaTask*>(a + p_craw);
  o.cta = reinterpret_cast<Sw16CtaTask*>(a + p_cta);
  o.cta_key = reinterpret_cast<ull*>(a + p_ck0);
  o.cta_key_alt = reinterpret_cast<ull*>(a + p_ck1);
  o.cta_idx = reinterpret_cast<uint32_t*>(a + p_ci0);
  o.cta_idx_alt = reinterpret_cast<uint32_t*>(a + p_ci1);
  o.n_cta = static_cast<uint32_t>(n_cta);
  // the rest of the preparation stays on the planner's stream (it reads the same
  // snapshot); the stream joins it before the plan's grids
  if (n_prof) dp_emit_kernel<<<gq32, 256, 0, s1>>>(in1, w, cls, o);
  if (n_cta) {
    cub::DoubleBuffer<ull> ck(o.cta_key, o.cta_key_alt);
    cub::DoubleBuffer<uint32_t> ci(o.cta_idx, o.cta_idx_alt);
    ST_CUDA(cub::DeviceRadixSort::SortPairs(a + p_tmp, t_lpt, ck, ci, static_cast<int>(n_cta), 0, 44 + 6, s1));
    o.cta_idx_sorted = ci.Current();
    dp_gather_cta_kernel<<<static_cast<uint32_t>((n_cta + 255) / 256), 256, 0, s1>>>(o);
  }
  uint2* zline = reinterpret_cast<uint2*>(a + p_z);
  dp_fill_zline_kernel<<<(zcols + 255) / 256, 256, 0, s1>>>(zline, zcols, pk_splat(-open));
  ST_CUDA(cudaGetLastError());
  c->launches += 3;
  ST_CUDA(cudaEventRecord(c->plan_ev, s1));
  ST_CUDA(cudaStreamWaitEvent(st, c->plan_ev, 0));

  plan->counters = counters;
  plan->counters_init = cinit;
  const DeviceDb db = db_view(c);
  const DeviceProfiles pv = prof_view(c);
  for (auto& cp : plan->classes) {
    Sw16Params& prm = cp.prm;
    prm.arena = db.arena;
    prm.prof = pv;
    prm.cta_tasks = o.cta + cta_begin[cp.cls];
    prm.n_cta_tasks = tot.n_cta[cp.cls];
    prm.warp_tasks = o.wt;
    prm.slots = o.slots;
    prm.scores = d_scores;
    prm.kernels = d_kernels;
    prm.ovf_count = counters + kNumClasses + 1;
    prm.ovf_pairs = w.list32;
    prm.work_counter = counters + cp.cls;
    prm.scratch = reinterpret_cast<uint2*>(a + cp.o_scratch);
    prm.zline = zline;
    prm.scratch_stride = cp.scratch_stride;
    prm.open = open;
    prm.ext = ext;
  }
  Sw32Params& p32 = plan->p32;
  p32.db = db;
  p32.prof = pv;
  p32.list = w.list32;
  p32.list_count = counters + kNumClasses + 1;
  p32.pair_query = w.pq;
  p32.pair_target = w.pt;
  p32.pair_center = w.pc;
  p32.pair_radius = w.pr;
  p32.scores = d_scores;
  p32.kernels = d_kernels;
  p32.work_counter = counters + kNumClasses;
  p32.scratch = reinterpret_cast<int2*>(a + p_s32);
  p32.scratch_stride = plan->scratch32_stride;
  p32.open = open;
  p32.ext = ext;
  p32.n_static = plan->n_static32;
  p32.band16 = (gaps16_ok(open, ext) && plan->n_static32 > 0) ? 1u : 0u;
  plan->kernels_per_run = static_cast<uint32_t>(plan->classes.size()) + 1 + p32.band16;
  tc.lap("stage 2 (enqueue)");
  if (trace_on())
    for (auto& cp : plan->classes)
      fprintf(stderr, "[st] dplan class %d: %u CTA tasks, %u warp tasks, grid %u, smem %u, scratch %u\n", cp.cls,
              tot.n_cta[cp.cls], tot.n_wt[cp.cls], cp.grid, cp.smem, cp.scratch_stride);
  *out = plan.release();
  return ST_OK;
}

// Batches of at least this many pairs are planned on the device
// (ST_DEVICE_PLAN=0 keeps the host planner for every size).
static bool use_device_plan(uint64_t n) {
  if (!env_u64("ST_DEVICE_PLAN", 1)) return false;
  return n >= env_u64("ST_DEVICE_PLAN_MIN", 16384);
}

// One batch of pairs in flight: its plan, device buffers, staging and the
// event after its result copies.
struct st_batch {
  st_ctx* c = nullptr;
  uint64_t n = 0;
  int32_t* scores = nullptr;
  uint32_t* kernels = nullptr;
  DevMem out, work;
  st_plan* plan = nullptr;
  std::unique_ptr<Pinned> stage;  // null when the caller's buffers are pinned
  cudaEvent_t done = nullptr;
  // with ST_TRACE: the stream reaching the batch, the plan's launches starting and ending, the download done
  cudaEvent_t tr[4] = {};
};

static void batch_release(st_batch* b) {
  st_ctx* c = b->c;
  for (auto& e : b->tr)
    if (e) {
      cudaEventSynchronize(e);
      cudaEventDestroy(e);
      e = nullptr;
    }
  if (b->done) {
    cudaEventSynchronize(b->done);
    c->spare_events.push_back(b->done);
  } else {
    cudaStreamSynchronize(c->stream);
  }
  if (b->plan) plan_free(b->plan);
  pool_put(c, std::move(b->out));
  pool_put(c, std::move(b->work));
  if (b->stage) c->pin_free.push_back(std::move(b->stage));
  delete b;
}

// Validates, uploads, plans and launches a batch and queues its result copies;
// does not wait for them. Batches of at least the device-plan size are planned
// on the GPU (one short wait for the per-class totals); smaller ones on the host.
static int batch_begin(st_ctx* c, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext, int32_t* scores,
                       uint32_t* kernels, st_batch** out) {
  std::unique_ptr<st_batch, void (*)(st_batch*)> b(new st_batch, batch_release);
  b->c = c;
  b->n = n;
  b->scores = scores;
  b->kernels = kernels;
  TraceClock tc("pairs");
  if (trace_on() && n) {
    if (!c->trace_base && cudaEventCreate(&c->trace_base) == cudaSuccess) cudaEventRecord(c->trace_base, c->stream);
    for (auto& e : b->tr) cudaEventCreate(&e);
    cudaEventRecord(b->tr[0], c->stream);
  }
  if (n == 0) {  // nothing to score: a batch that is done when the stream gets there
    ST_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
    ST_CUDA(cudaEventRecord(b->done, c->stream));
    *out = b.release();
    return ST_OK;
  }
  ST_TRY(pool_get(c, n * 8, b->out));
  int32_t* d_scores = b->out.as<int32_t>();
  uint32_t* d_kern = reinterpret_cast<uint32_t*>(d_scores + n);
  // Results come back through pinned memory unless the caller's buffers are
  // pinned already.
  int32_t* h_scores = scores;
  uint32_t* h_kern = kernels;
  if (!(host_pinned(scores) && (!kernels || host_pinned(kernels)))) {
    for (size_t i = 0; i < c->pin_free.size(); ++i)
      if (c->pin_free[i]->bytes >= n * 8) {
        b->stage = std::move(c->pin_free[i]);
        c->pin_free.erase(c->pin_free.begin() + i);
        break;
      }
    if (!b->stage) b->stage.reset(new Pinned);
    ST_TRY(b->stage->reserve(n * 8));
    h_scores = b->stage->as<int32_t>();
    h_kern = kernels ? b->stage->as<uint32_t>(n * 4) : nullptr;
  }
  if (use_device_plan(n)) {
    uint32_t max_len = 0, max_m = 0;
    ST_TRY(validate_pairs(c, pairs, n, &max_len, &max_m));
    ST_TRY(sync_profiles(c));
    tc.lap("validate");
    ST_TRY(dplan_build(c, pairs, n, open, ext, d_scores, d_kern, max_len, max_m, b->work, &b->plan));
  } else {
    ST_TRY(plan_build(c, pairs, n, open, ext, d_scores, d_kern, &b->plan, false, c->stream, 0));
    tc.lap("plan");
  }
  if (b->tr[1]) cudaEventRecord(b->tr[1], c->stream);
  ST_TRY(plan_run(b->plan));
  if (b->tr[2]) cudaEventRecord(b->tr[2], c->stream);
  ST_CUDA(cudaMemcpyAsync(h_scores, d_scores, n * 4, cudaMemcpyDeviceToHost, c->stream));
  if (kernels) ST_CUDA(cudaMemcpyAsync(h_kern, d_kern, n * 4, cudaMemcpyDeviceToHost, c->stream));
  if (b->tr[3]) cudaEventRecord(b->tr[3], c->stream);
  if (!c->spare_events.empty()) {
    b->done = c->spare_events.back();
    c->spare_events.pop_back();
  } else {
    ST_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
  }
  ST_CUDA(cudaEventRecord(b->done, c->stream));
  *out = b.release();
  return ST_OK;
}

// Waits for a batch, writes its results to the caller's buffers and releases it.
static int batch_finish(st_batch* b) {
  TraceClock tc("pairs");
  st_ctx* c = b->c;
  const cudaError_t e = cudaEventSynchronize(b->done);
  if (e == cudaSuccess && b->tr[3] && c->trace_base) {
    float t[4] = {};
    for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&t[i], c->trace_base, b->tr[i]);
    fprintf(stderr, "[st] batch device: stream at %.3f, plan launches %.3f - %.3f, download done %.3f ms\n", t[0], t[1],
            t[2], t[3]);
  }
  if (e == cudaSuccess && b->stage) {
    const uint64_t n = b->n;
    const int32_t* hs = b->stage->as<int32_t>();
    const uint32_t* hk = b->stage->as<uint32_t>(n * 4);
    int32_t* scores = b->scores;
    uint32_t* kernels = b->kernels;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < static_cast<int64_t>((n + 262143) / 262144); ++k) {
      const uint64_t a0 = static_cast<uint64_t>(k) * 262144, a1 = std::min<uint64_t>(n, a0 + 262144);
      memcpy(scores + a0, hs + a0, (a1 - a0) * 4);
      if (kernels) memcpy(kernels + a0, hk + a0, (a1 - a0) * 4);
    }
  }
  batch_release(b);
  (void)c;
  tc.lap("wait+copy");
  if (e != cudaSuccess) return fail(ST_ECUDA, "batch failed: %s", cudaGetErrorString(e));
  return ST_OK;
}

extern "C" int st_sw_score_pairs_async(st_ctx* c, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext,
                                       int32_t* scores, uint32_t* kernels, st_batch** batch) {
  CTX_GUARD(c);
  if (!batch || (n && (!pairs || !scores))) return fail(ST_EINVAL, "st_sw_score_pairs_async: null argument");
  *batch = nullptr;
  return batch_begin(c, pairs, n, open, ext, scores, kernels, batch);
}

extern "C" int st_batch_wait(st_batch* batch) {
  if (!batch) return fail(ST_EINVAL, "st_batch_wait: null batch");
  st_ctx* c = batch->c;
  if (batch->done) {  // wait without holding the context, so other threads can use it meanwhile
    cudaSetDevice(c->device);
    cudaEventSynchronize(batch->done);
  }
  CTX_GUARD(c);
  return batch_finish(batch);
}

extern "C" int st_batch_query(st_batch* batch) {
  if (!batch) return fail(ST_EINVAL, "st_batch_query: null batch");
  if (!batch->done) return ST_OK;
  cudaSetDevice(batch->c->device);
  const cudaError_t e = cudaEventQuery(batch->done);
  if (e == cudaSuccess) return ST_OK;
  if (e == cudaErrorNotReady) {
    cudaGetLastError();
    return 1;
  }
  return fail(ST_ECUDA, "batch failed: %s", cudaGetErrorString(e));
}

extern "C" int st_sw_score_pairs(st_ctx* c, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext,
                                 int32_t* scores, uint32_t* kernels) {
  CTX_GUARD(c);
  if (n && (!pairs || !scores)) return fail(ST_EINVAL, "st_sw_score_pairs: null argument");
  if (n == 0) return ST_OK;
  if (use_device_plan(n) || pipeline_bounds(n).size() <= 2) {
    st_batch* b = nullptr;
    ST_TRY(batch_begin(c, pairs, n, open, ext, scores, kernels, &b));
    return batch_finish(b);
  }
  // large batches with the host planner: pipelined chunks
  DevMem d_out;
  ST_TRY(pool_get(c, n * 8, d_out));
  struct Back {
    st_ctx* c;
    DevMem* m;
    ~Back() { pool_put(c, std::move(*m)); }
  } back{c, &d_out};
  int32_t* d_scores = d_out.as<int32_t>();
  uint32_t* d_kern = reinterpret_cast<uint32_t*>(d_scores + n);
  TraceClock tc("pairs");
  const bool direct = host_pinned(scores) && (!kernels || host_pinned(kernels));
  int32_t* h_scores = scores;
  uint32_t* h_kern = kernels;
  if (!direct) {
    ST_TRY(c->out_pin.reserve(n * 8));
    h_scores = c->out_pin.as<int32_t>();
    h_kern = kernels ? c->out_pin.as<uint32_t>(n * 4) : nullptr;
  }
  auto copy_out = [&]() {
    if (direct) return;
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < static_cast<int64_t>((n + 262143) / 262144); ++b) {
      const uint64_t a0 = static_cast<uint64_t>(b) * 262144, a1 = std::min<uint64_t>(n, a0 + 262144);
      memcpy(scores + a0, h_scores + a0, (a1 - a0) * 4);
      if (kernels) memcpy(kernels + a0, h_kern + a0, (a1 - a0) * 4);
    }
  };
  const std::vector<uint64_t> bounds = pipeline_bounds(n);
  const uint64_t chunks = bounds.size() - 1;
  // Pipelined: the pairs are cut into contiguous chunks, each planned on the
  // host while the chunks before it run. Chunks alternate between two side
  // streams, so the tail of one chunk's persistent grid overlaps the start of
  // the next; each chunk downloads its own scores on its stream.
  ST_TRY(sync_profiles(c));
  {
    // every pair is checked before the first chunk launches, so an error leaves no partial work
    const uint32_t n_prof = static_cast<uint32_t>(c->profs.size());
    int64_t bad = INT64_MAX;
#pragma omp parallel for schedule(static) reduction(min : bad)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
      const st_pair& p = pairs[i];
      if (p.profile >= n_prof || !c->profs[p.profile].live || p.target >= c->n_seqs) bad = std::min<int64_t>(bad, i);
    }
    if (bad != INT64_MAX) {
      const st_pair& p = pairs[bad];
      if (p.profile >= n_prof || !c->profs[p.profile].live)
        return fail(ST_EINVAL, "pair %lld: unknown profile id %u", static_cast<long long>(bad), p.profile);
      return fail(ST_EINVAL, "pair %lld: target %u outside the database (%u sequences)", static_cast<long long>(bad),
                  p.target, c->n_seqs);
    }
  }
  const int n_side = pipeline_streams();
  for (int i = 0; i < n_side; ++i)
    if (!c->side[i]) ST_CUDA(cudaStreamCreateWithFlags(&c->side[i], cudaStreamNonBlocking));
  for (auto& e : c->side_ev)
    if (!e) ST_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  ST_CUDA(cudaEventRecord(c->side_ev[0], c->stream));  // after earlier work on the caller's stream
  for (int i = 0; i < n_side; ++i) ST_CUDA(cudaStreamWaitEvent(c->side[i], c->side_ev[0], 0));
  std::vector<std::unique_ptr<st_plan, void (*)(st_plan*)>> plans;
  plans.reserve(chunks);
  // with ST_TRACE: device time of each chunk's launches, relative to the batch start
  std::vector<cudaEvent_t> tev;
  if (trace_on()) {
    tev.assign(2 * chunks + 1, nullptr);
    for (auto& e : tev) cudaEventCreate(&e);
    cudaEventRecord(tev[0], c->stream);
  }
  struct Drain {  // on every exit: the side streams finish before any plan (and its arena) is released
    st_ctx* c;
    ~Drain() {
      for (auto s : c->side)
        if (s) cudaStreamSynchronize(s);
    }
  };
  int rc = ST_OK;
  {
    Drain drain{c};
    for (uint64_t k = 0; k < chunks && rc == ST_OK; ++k) {
      const uint64_t b = bounds[k], e = bounds[k + 1];
      cudaStream_t s = c->side[k % n_side];
      st_plan* p = nullptr;
      rc = plan_build(c, pairs + b, e - b, open, ext, d_scores + b, d_kern + b, &p, false, s,
                      static_cast<int>(k % st_ctx::kStageRing));
      if (rc != ST_OK) break;
      plans.emplace_back(p, plan_free);
      if (!tev.empty()) cudaEventRecord(tev[1 + 2 * k], s);
      st_ctx::ForkSet* fs = nullptr;
      rc = fork_set(c, 1 + static_cast<int>(k % n_side), &fs);
      if (rc != ST_OK) break;
      if (plan_enqueue(p, s, fs) != ST_OK) {
        rc = fail(ST_ECUDA, "plan launch failed: %s", cudaGetErrorString(cudaGetLastError()));
        break;
      }
      c->launches += p->kernels_per_run;
      if (!tev.empty()) cudaEventRecord(tev[2 + 2 * k], s);
      if (cudaMemcpyAsync(h_scores + b, d_scores + b, (e - b) * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          (kernels && cudaMemcpyAsync(h_kern + b, d_kern + b, (e - b) * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess))
        rc = fail(ST_ECUDA, "score download failed: %s", cudaGetErrorString(cudaGetLastError()));
      tc.lap("chunk");
    }
    if (rc == ST_OK) {
      // the caller's stream is ordered after the batch
      for (int i = 0; i < n_side && rc == ST_OK; ++i)
        if (cudaEventRecord(c->side_ev[1 + i], c->side[i]) != cudaSuccess ||
            cudaStreamWaitEvent(c->stream, c->side_ev[1 + i], 0) != cudaSuccess)
          rc = fail(ST_ECUDA, "stream ordering failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
  }
  if (!tev.empty()) {
    cudaStreamSynchronize(c->stream);
    for (uint64_t k = 0; k < plans.size(); ++k) {
      float a = 0, b = 0;
      cudaEventElapsedTime(&a, tev[0], tev[1 + 2 * k]);
      cudaEventElapsedTime(&b, tev[0], tev[2 + 2 * k]);
      fprintf(stderr, "[st] chunk %llu device %.3f .. %.3f ms (%.3f)\n", static_cast<unsigned long long>(k), a, b, b - a);
    }
    for (auto e : tev) cudaEventDestroy(e);
  }
  if (rc != ST_OK) return rc;
  ST_CUDA(cudaStreamSynchronize(c->stream));
  copy_out();
  tc.lap("run+download");
  return ST_OK;
}

// ---------------------------------------------------------------------------
// end cells and alignment spans (sw_score_end_with + the reverse pass of
// align_canonical), exact 32-bit kernel
// ---------------------------------------------------------------------------
// Scores n pairs (targets in `db`, unbanded) in end mode and, with `span`,
// runs the reverse pass from each end cell. Outputs go to host buffers:
// scores[i]; ends[2i..2i+1] = (query end, target end); with span,
// starts[2i..2i+1] = (query start, target start); -1 where the score is 0.
static int end_pairs_run(st_ctx* c, const DeviceDb& db, const uint32_t* pq_h, const uint32_t* pt_h, uint64_t n,
                         uint32_t max_m, uint32_t max_len, int32_t open, int32_t ext, bool span, int32_t* scores,
                         int32_t* ends, int32_t* starts) {
  if (n == 0) return ST_OK;
  if (n > 0xFFFFFFF0ull) return fail(ST_EINVAL, "too many pairs");
  uint32_t grid = 0;
  const uint32_t sstride = max_m > static_cast<uint32_t>(kSw32Rows) ? max_len : 0;
  ST_TRY(grid_sw32(c, n, n, sstride, &grid));
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    const size_t o = off;
    off = (off + bytes + 255) & ~static_cast<size_t>(255);
    return o;
  };
  const size_t o_pq = carve(n * 4), o_pt = carve(n * 4), o_zero = carve(n * 4), o_list = carve(n * 4),
               o_cnt = carve(16), o_s = carve(n * 4), o_eq = carve(n * 4), o_et = carve(n * 4), o_rs = carve(n * 4),
               o_sq = carve(n * 4), o_st = carve(n * 4),
               o_scr = carve(sstride ? static_cast<size_t>(grid) * kWarps32 * sstride * sizeof(int2) : 16);
  const size_t up_bytes = o_zero;  // pq, pt travel in one copy
  DevMem a;
  ST_TRY(pool_get(c, off, a));
  struct Back {
    st_ctx* c;
    DevMem* m;
    ~Back() { pool_put_after(c, std::move(*m), c->stream); }
  } back{c, &a};
  char* d = a.as<char>();
  ST_TRY(c->pin.reserve(up_bytes + 16));
  ST_CUDA(cudaStreamSynchronize(c->stream));  // the pinned block may still feed an earlier copy
  char* h = c->pin.as<char>();
  memcpy(h + o_pq, pq_h, n * 4);
  memcpy(h + o_pt, pt_h, n * 4);
  ST_CUDA(cudaMemcpyAsync(d, h, up_bytes, cudaMemcpyHostToDevice, c->stream));
  ST_CUDA(cudaMemsetAsync(d + o_zero, 0, n * 4, c->stream));
  ST_CUDA(cudaMemsetAsync(d + o_cnt, 0, 16, c->stream));
  uint32_t* cnt = reinterpret_cast<uint32_t*>(d + o_cnt);  // [0] list count, [1], [2] work counters
  const uint32_t n32 = static_cast<uint32_t>(n);
  ST_CUDA(cudaMemcpyAsync(cnt, &n32, 4, cudaMemcpyHostToDevice, c->stream));
  dp_iota_kernel<<<static_cast<uint32_t>(std::min<uint64_t>((n + 255) / 256, 65535)), 256, 0, c->stream>>>(
      reinterpret_cast<uint32_t*>(d + o_list), n32);
  Sw32Params p{};
  p.db = db;
  p.prof = prof_view(c);
  p.list = reinterpret_cast<const uint32_t*>(d + o_list);
  p.list_count = cnt;
  p.pair_query = reinterpret_cast<const uint32_t*>(d + o_pq);
  p.pair_target = reinterpret_cast<const uint32_t*>(d + o_pt);
  p.pair_center = reinterpret_cast<const int32_t*>(d + o_zero);
  p.pair_radius = reinterpret_cast<const int32_t*>(d + o_zero);  // unused in the end modes
  p.scores = reinterpret_cast<int32_t*>(d + o_s);
  p.kernels = nullptr;
  p.work_counter = cnt + 1;
  p.scratch = reinterpret_cast<int2*>(d + o_scr);
  p.scratch_stride = sstride;
  p.open = open;
  p.ext = ext;
  p.end_q = reinterpret_cast<int32_t*>(d + o_eq);
  p.end_t = reinterpret_cast<int32_t*>(d + o_et);
  sw32_end_kernel<kWarps32, kSw32End><<<grid, kWarps32 * 32, 0, c->stream>>>(p);
  c->launches += 2;
  if (span) {
    Sw32Params r = p;
    r.rev_q = p.end_q;
    r.rev_t = p.end_t;
    r.scores = reinterpret_cast<int32_t*>(d + o_rs);
    r.end_q = reinterpret_cast<int32_t*>(d + o_sq);
    r.end_t = reinterpret_cast<int32_t*>(d + o_st);
    r.work_counter = cnt + 2;
    sw32_end_kernel<kWarps32, kSw32RevEnd><<<grid, kWarps32 * 32, 0, c->stream>>>(r);
    ++c->launches;
  }
  ST_CUDA(cudaGetLastError());
  std::vector<int32_t> eq(n), et(n), rs, sq, st;
  ST_CUDA(cudaMemcpyAsync(scores, d + o_s, n * 4, cudaMemcpyDeviceToHost, c->stream));
  ST_CUDA(cudaMemcpyAsync(eq.data(), d + o_eq, n * 4, cudaMemcpyDeviceToHost, c->stream));
  ST_CUDA(cudaMemcpyAsync(et.data(), d + o_et, n * 4, cudaMemcpyDeviceToHost, c->stream));
  if (span) {
    rs.resize(n);
    sq.resize(n);
    st.resize(n);
    ST_CUDA(cudaMemcpyAsync(rs.data(), d + o_rs, n * 4, cudaMemcpyDeviceToHost, c->stream));
    ST_CUDA(cudaMemcpyAsync(sq.data(), d + o_sq, n * 4, cudaMemcpyDeviceToHost, c->stream));
    ST_CUDA(cudaMemcpyAsync(st.data(), d + o_st, n * 4, cudaMemcpyDeviceToHost, c->stream));
  }
  ST_CUDA(cudaStreamSynchronize(c->stream));
  for (uint64_t i = 0; i < n; ++i) {
    ends[2 * i] = eq[i];
    ends[2 * i + 1] = et[i];
    if (!span) continue;
    if (scores[i] > 0 && rs[i] != scores[i])  // impossible: the best alignment ending at the end cell lies in the prefix
      return fail(ST_ECUDA, "pair %llu: reverse pass scored %d, forward %d", static_cast<unsigned long long>(i),
                  rs[i], scores[i]);
    starts[2 * i] = scores[i] > 0 ? eq[i] - sq[i] : -1;
    starts[2 * i + 1] = scores[i] > 0 ? et[i] - st[i] : -1;
  }
  return ST_OK;
}

static int end_pairs_entry(st_ctx* c, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext, bool span,
                           int32_t* scores, int32_t* ends, int32_t* starts) {
  if (n && (!pairs || !scores || !ends || (span && !starts))) return fail(ST_EINVAL, "null argument");
  if (!c->has_db) return fail(ST_ESTATE, "no target database uploaded (st_db_upload)");
  uint32_t max_len = 0, max_m = 0;
  ST_TRY(validate_pairs(c, pairs, n, &max_len, &max_m));
  std::vector<uint32_t> pq(n), pt(n);
  for (uint64_t i = 0; i < n; ++i) {
    if (pairs[i].band_radius >= 0)
      return fail(ST_EINVAL, "pair %llu: end cells are defined for full local alignments (band_radius < 0)",
                  static_cast<unsigned long long>(i));
    pq[i] = pairs[i].profile;
    pt[i] = pairs[i].target;
  }
  ST_TRY(sync_profiles(c));
  return end_pairs_run(c, db_view(c), pq.data(), pt.data(), n, max_m, max_len, open, ext, span, scores, ends, starts);
}

extern "C" int st_sw_score_end_pairs(st_ctx* c, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext,
                                     int32_t* scores, int32_t* ends) {
  CTX_GUARD(c);
  return end_pairs_entry(c, pairs, n, open, ext, false, scores, ends, nullptr);
}

extern "C" int st_sw_score_end(st_ctx* c, uint32_t profile, const uint8_t* target, uint32_t n, int32_t open,
                               int32_t ext, int32_t* score, int32_t* q_end, int32_t* t_end) {
  CTX_GUARD(c);
  if (!score || !q_end || !t_end || (n && !target)) return fail(ST_EINVAL, "st_sw_score_end: null argument");
  ST_TRY(check_profile(c, profile));
  ST_TRY(sync_profiles(c));
  const uint32_t m = c->profs[profile].m;
  if (m == 0 || n == 0) {  // src/simd.rs:302-304
    *score = 0;
    *q_end = *t_end = -1;
    return ST_OK;
  }
  // the target as a one-sequence database in a pooled device block
  const size_t tb = up16(n) + 16;
  std::vector<uint8_t> h(tb + 16, kSentinel);
  for (uint32_t i = 0; i < n; ++i) h[i] = target[i] < kSentinel ? target[i] : kSentinel;
  const uint64_t zero = 0;
  memcpy(h.data() + tb, &zero, 8);
  memcpy(h.data() + tb + 8, &n, 4);
  DevMem a;
  ST_TRY(pool_get(c, h.size(), a));
  struct Back {
    st_ctx* c;
    DevMem* m;
    ~Back() { pool_put_after(c, std::move(*m), c->stream); }
  } back{c, &a};
  ST_CUDA(cudaMemcpyAsync(a.p, h.data(), h.size(), cudaMemcpyHostToDevice, c->stream));
  DeviceDb db;
  db.arena = a.as<uint8_t>();
  db.offset = reinterpret_cast<const uint64_t*>(a.as<char>() + tb);
  db.length = reinterpret_cast<const uint32_t*>(a.as<char>() + tb + 8);
  db.n_seqs = 1;
  const uint32_t t0 = 0;
  int32_t ends[2];
  ST_TRY(end_pairs_run(c, db, &profile, &t0, 1, m, n, open, ext, false, score, ends, nullptr));
  *q_end = ends[0];
  *t_end = ends[1];
  return ST_OK;
}

extern "C" int st_sw_align_span_pairs(st_ctx* c, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext,
                                      int32_t* scores, int32_t* ends, int32_t* starts) {
  CTX_GUARD(c);
  return end_pairs_entry(c, pairs, n, open, ext, true, scores, ends, starts);
}

// ---------------------------------------------------------------------------
// plain per-call SW (one pair, one launch of each kernel, blocking)
// ---------------------------------------------------------------------------
// One per-call scoring on slot `sl`, in two phases.  sw_score_prepare runs under the context lock: the
// checks, the profile tables, the sizes, the slot's buffers (device memory is accounted to the context) and,
// when profiles changed since the slot's last call, the event that orders the call after the context
// stream's work so far.  sw_score_launch runs outside it, on the slot's own stream: the staged inputs, the
// copy and the launches.  Between the two the call holds the context's call lock shared, so the profile
// tables it captured cannot be reallocated under it (table growth takes that lock exclusively, then waits
// for the calls' streams).
struct SwCall {
  uint32_t profile = 0, n = 0, k = 0, P = 1, rows = 0, ncols = 0, sstride = 0;
  int32_t open = 0, ext = 0;
  bool use16 = false, wait = false;
  size_t tbytes = 0, o_off = 0, o_len = 0, o_pt = 0, o_pq = 0, o_pc = 0, o_pr = 0, o_cta = 0, o_wt = 0, o_slots = 0,
         o_cnt = 0, o_list = 0, o_zline = 0, total = 0;
  DeviceProfiles pv;
};

// *launch says whether there is work to launch (an empty query or target scores 0 at once).
static int sw_score_prepare(st_ctx* c, CallSlot* sl, uint32_t profile, uint32_t n, int32_t open, int32_t ext,
                            int32_t* score, uint32_t* kernel, SwCall* w, bool* launch) {
  *launch = false;
  ST_TRY(check_profile(c, profile));
  ST_TRY(sync_profiles(c));
  const ProfileMeta& pm = c->profs[profile];
  if (pm.m == 0 || n == 0) {  // src/simd.rs:253-255
    *score = 0;
    if (kernel) *kernel = ST_KERNEL_NONE;
    return ST_OK;
  }
  // staging block (one host->device copy per call):
  //   [target codes, padded] [db offset u64] [db length u32] [pair: target u32, query u32, center i32, radius i32]
  //   [cta task] [warp task] [slots x64] [counters x(kNumClasses+2)] [32-bit list u32] [first-pass boundary]
  // and, behind it in the pinned block only, the score and kernel tag the kernels write
  w->profile = profile;
  w->n = n;
  w->open = open;
  w->ext = ext;
  w->tbytes = up16(n) + 32;
  size_t o = w->tbytes;
  w->o_off = o; o += 8;
  w->o_len = o; o += 4;
  w->o_pt = o; o += 4;
  w->o_pq = o; o += 4;
  w->o_pc = o; o += 4;
  w->o_pr = o; o += 4;
  o = up16(o);
  w->o_cta = o; o += sizeof(Sw16CtaTask);
  w->o_wt = o; o += sizeof(Sw16WarpTask);
  o = up16(o);  // slot records are read as 16-byte vectors
  w->o_slots = o; o += 64 * sizeof(Sw16Slot);
  w->o_cnt = o; o += (kNumClasses + 2) * 4;
  w->o_list = o; o += 4;
  o = up16(o);
  w->o_zline = o; o += (static_cast<size_t>(std::max<uint32_t>(32, static_cast<uint32_t>(up16(n)))) +
                        static_cast<size_t>(32 * 4 + 16)) * sizeof(uint2);
  w->total = up16(o);
  w->use16 = pm.fits8 && gaps16_ok(open, ext);
  w->k = 0;
  w->P = 1;
  w->rows = 0;
  if (w->use16) {
    w->k = static_cast<uint32_t>(tuning_pick_single(&c->tuning, pm.m, n));
    w->rows = kClasses[w->k].G * kClasses[w->k].R;
    w->P = (pm.m + w->rows - 1) / w->rows;
    if (static_cast<size_t>(kProfRows) * w->P * w->rows > static_cast<size_t>(g_class_smem[w->k]))
      return fail(ST_EINVAL, "query of %u rows too long for the shared-memory profile", pm.m);
  }
  w->ncols = std::max<uint32_t>(32, static_cast<uint32_t>(up4(n)));
  if (w->use16 && w->P > 1)
    w->ncols = std::max<uint32_t>(w->ncols, static_cast<uint32_t>(up16(kClasses[w->k].C * kClasses[w->k].G)));
  w->sstride = std::max<uint32_t>(w->ncols, static_cast<uint32_t>(up16(n) + 32));
  // any warp of the CTA may take the task: room for every group of the CTA
  const size_t scratch_need = static_cast<size_t>(kClasses[w->k].W) * 8 * w->sstride * sizeof(uint2);
  if (!sl->s) {
    ST_CUDA(cudaStreamCreateWithFlags(&sl->s, cudaStreamNonBlocking));
    ST_CUDA(cudaEventCreateWithFlags(&sl->ev_in, cudaEventDisableTiming));
    ST_CUDA(cudaEventCreateWithFlags(&sl->ev_done, cudaEventDisableTiming));
  }
  // the slot's previous call has been waited for, so its pinned block and device buffers are free
  ST_TRY(sl->pin.reserve(w->total + 16));
  if (sl->stage.bytes < w->total) ST_TRY(dev_alloc(&c->mt, sl->stage, w->total * 2));
  if (sl->scratch.bytes < scratch_need) ST_TRY(dev_alloc(&c->mt, sl->scratch, scratch_need * 2));
  w->pv = prof_view(c);
  // the profile tables and layouts are written in the context stream's order: unless none changed since the
  // slot's last call (its stream is ordered after that point already), start after the stream's work so far
  w->wait = sl->epoch != c->prof_epoch;
  if (w->wait) {
    ST_CUDA(cudaEventRecord(sl->ev_in, c->stream));
    sl->epoch = c->prof_epoch;
  }
  c->launches += w->use16 ? 2 : 1;
  *launch = true;
  return ST_OK;
}

// The call's inputs staged and uploaded and its kernels launched; they write the score and kernel tag
// straight into the slot's pinned block at *res_off (pinned memory is device-accessible under unified
// addressing, so no copy back is queued), and ev_done marks their arrival.
static int sw_score_launch(CallSlot* sl, const uint8_t* target, const SwCall& w, size_t* res_off) {
  const uint32_t n = w.n;
  char* h = sl->pin.as<char>();
  memset(h, 0, w.total);
  for (uint32_t i = 0; i < n; ++i) h[i] = static_cast<char>(target[i] < kSentinel ? target[i] : kSentinel);
  memset(h + n, kSentinel, w.tbytes - n);
  *reinterpret_cast<uint64_t*>(h + w.o_off) = 0;
  *reinterpret_cast<uint32_t*>(h + w.o_len) = n;
  *reinterpret_cast<uint32_t*>(h + w.o_pt) = 0;
  *reinterpret_cast<uint32_t*>(h + w.o_pq) = w.profile;
  *reinterpret_cast<int32_t*>(h + w.o_pc) = 0;
  *reinterpret_cast<int32_t*>(h + w.o_pr) = -1;  // no band
  Sw16CtaTask ct{w.profile, 0, 1, w.P * std::max<uint32_t>(w.rows, 1)};
  Sw16WarpTask wt{0, w.ncols};
  memcpy(h + w.o_cta, &ct, sizeof(ct));
  memcpy(h + w.o_wt, &wt, sizeof(wt));
  Sw16Slot* slots = reinterpret_cast<Sw16Slot*>(h + w.o_slots);
  for (int s = 0; s < 64; ++s) slots[s] = Sw16Slot{kNoPair, 0, 0, 0};
  slots[0] = Sw16Slot{0, 0, static_cast<uint32_t>(up16(n)), n};  // the staged target sits at offset 0
  uint32_t* cnt = reinterpret_cast<uint32_t*>(h + w.o_cnt);
  if (!w.use16) cnt[kNumClasses + 1] = 1;  // the pair goes straight to the 32-bit list
  *reinterpret_cast<uint32_t*>(h + w.o_list) = 0;
  {
    uint2* z = reinterpret_cast<uint2*>(h + w.o_zline);
    const size_t nz = (w.total - w.o_zline) / sizeof(uint2);
    for (size_t i = 0; i < nz; ++i) z[i] = make_uint2(0u, pk_splat(-w.open));
  }
  *res_off = w.total;
  int32_t* h_res = sl->pin.as<int32_t>(*res_off);
  h_res[0] = 0;
  h_res[1] = 0;
  char* d = sl->stage.as<char>();
  cudaStream_t st = sl->s;
  if (w.wait) ST_CUDA(cudaStreamWaitEvent(st, sl->ev_in, 0));
  ST_CUDA(cudaMemcpyAsync(d, h, w.total, cudaMemcpyHostToDevice, st));
  DeviceDb db;
  db.arena = reinterpret_cast<const uint8_t*>(d);
  db.offset = reinterpret_cast<const uint64_t*>(d + w.o_off);
  db.length = reinterpret_cast<const uint32_t*>(d + w.o_len);
  db.n_seqs = 1;
  uint32_t* d_cnt = reinterpret_cast<uint32_t*>(d + w.o_cnt);
  int32_t* d_score = h_res;
  uint32_t* d_kern = reinterpret_cast<uint32_t*>(h_res + 1);
  uint32_t* d_list = reinterpret_cast<uint32_t*>(d + w.o_list);
  if (w.use16) {
    Sw16Params prm;
    prm.arena = reinterpret_cast<const uint8_t*>(d);
    prm.prof = w.pv;
    prm.cta_tasks = reinterpret_cast<const Sw16CtaTask*>(d + w.o_cta);
    prm.n_cta_tasks = 1;
    prm.warp_tasks = reinterpret_cast<const Sw16WarpTask*>(d + w.o_wt);
    prm.slots = reinterpret_cast<const Sw16Slot*>(d + w.o_slots);
    prm.scores = d_score;
    prm.kernels = d_kern;
    prm.ovf_count = d_cnt + kNumClasses + 1;
    prm.ovf_pairs = d_list;
    prm.work_counter = d_cnt + w.k;
    prm.scratch = sl->scratch.as<uint2>();
    prm.zline = reinterpret_cast<const uint2*>(d + w.o_zline);
    prm.scratch_stride = w.sstride;
    prm.open = w.open;
    prm.ext = w.ext;
    kClasses[w.k].fn<<<1, kClasses[w.k].W * 32, kProfRows * w.P * w.rows, st>>>(prm);
  }
  // the 32-bit kernel scores the pair only when it is in the list (headroom reached, or not 16-bit eligible)
  Sw32Params p32;
  p32.db = db;
  p32.prof = w.pv;
  p32.list = d_list;
  p32.list_count = d_cnt + kNumClasses + 1;
  p32.pair_query = reinterpret_cast<const uint32_t*>(d + w.o_pq);
  p32.pair_target = reinterpret_cast<const uint32_t*>(d + w.o_pt);
  p32.pair_center = reinterpret_cast<const int32_t*>(d + w.o_pc);
  p32.pair_radius = reinterpret_cast<const int32_t*>(d + w.o_pr);
  p32.scores = d_score;
  p32.kernels = d_kern;
  p32.work_counter = d_cnt + kNumClasses;
  p32.scratch = reinterpret_cast<int2*>(sl->scratch.p);
  p32.scratch_stride = static_cast<uint32_t>(up16(n) + 32);
  p32.open = w.open;
  p32.ext = w.ext;
  sw32_kernel<kWarps32><<<1, kWarps32 * 32, 0, st>>>(p32);
  ST_CUDA(cudaGetLastError());
  ST_CUDA(cudaEventRecord(sl->ev_done, st));
  return ST_OK;
}

// The plain per-call drop-in for sw_score_with.  Calls from several host threads proceed at once: each
// takes a call slot (its own stream and buffers), holds the context lock only while it checks and sizes
// the call, stages and launches on its own stream outside that lock, and waits for its result.
extern "C" int st_sw_score(st_ctx* c, uint32_t profile, const uint8_t* target, uint32_t n, int32_t open, int32_t ext,
                           int32_t* score, uint32_t* kernel) {
  if (!c) return fail(ST_EINVAL, "null context");
  if (!score || (n && !target)) return fail(ST_EINVAL, "st_sw_score: null argument");
  CallSlot* sl = call_acquire(c);
  SwCall w;
  bool launch = false, queued = false;
  size_t res_off = 0;
  int rc;
  std::shared_lock<std::shared_mutex> tables;  // the profile tables stay while this call's work is enqueued
  {
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    rc = cudaSetDevice(c->device) == cudaSuccess ? ST_OK : fail(ST_ECUDA, "cudaSetDevice(%d) failed", c->device);
    if (rc == ST_OK) rc = sw_score_prepare(c, sl, profile, n, open, ext, score, kernel, &w, &launch);
    if (rc == ST_OK && launch) tables = std::shared_lock<std::shared_mutex>(c->call_rw);
  }
  if (rc == ST_OK && launch) {
    rc = sw_score_launch(sl, target, w, &res_off);
    queued = rc == ST_OK;
  }
  if (tables.owns_lock()) tables.unlock();
  if (queued) {
    const cudaError_t e = cudaEventSynchronize(sl->ev_done);
    if (e != cudaSuccess) {
      rc = fail(ST_ECUDA, "st_sw_score: %s", cudaGetErrorString(e));
    } else {
      const int32_t* res = sl->pin.as<int32_t>(res_off);
      *score = res[0];
      if (kernel) *kernel = static_cast<uint32_t>(res[1]);
    }
  } else if (launch && sl->s) {
    cudaStreamSynchronize(sl->s);  // a failed launch phase: let whatever was queued finish before the slot's reuse
    cudaGetLastError();
    sl->epoch = 0;  // its stream may not have waited for the context stream: the next call waits again
  }
  call_release(c, sl);
  return rc;
}

// ---------------------------------------------------------------------------
// ungapped
// ---------------------------------------------------------------------------
static uint32_t ung_stride(st_ctx* c) { return static_cast<uint32_t>(up16(c->max_m) + 32); }

// max_m: the longest query the jobs refer to (0: any live profile), which sizes
// the staged profile rows and so the CTAs that fit on an SM.
static int launch_ungapped(st_ctx* c, bool hits, const void* d_jobs, uint64_t n, int32_t* d_out, uint32_t max_m = 0) {
  if (n == 0) return ST_OK;
  UngappedParams prm;
  prm.db = db_view(c);
  prm.prof = prof_view(c);
  prm.jobs = d_jobs;
  prm.n = n;
  prm.out = d_out;
  prm.max_m_pad = max_m ? static_cast<uint32_t>(up16(max_m) + 32) : ung_stride(c);
  const size_t smem = 16 + static_cast<size_t>(kProfRows) * prm.max_m_pad + 16;
  if (smem > static_cast<size_t>(g_ung_smem))
    return fail(ST_EINVAL, "query too long for the ungapped kernel (%u rows)", max_m ? max_m : c->max_m);
  const uint64_t grid = (n + kUngChunk - 1) / kUngChunk;
  if (grid > 0x7FFFFFFFull) return fail(ST_EINVAL, "too many ungapped jobs");
  // hit lists: one hit per lane with refill; with ST_UNGAPPED_SPLIT=1 the form that splits a run's work evenly
  // over the lanes (measured slower on 2x10^7 hits: 2.33 against 1.68 ms; its static shared memory halves the
  // CTAs per SM and its phases add barriers)
  const bool split = env_u64("ST_UNGAPPED_SPLIT", 0) != 0;
  if (hits && split && smem <= static_cast<size_t>(g_ung_split_smem))
    ungapped_hits_split_kernel<<<static_cast<uint32_t>(grid), kUngSplitLanes, smem, c->stream>>>(prm);
  else if (hits)
    ungapped_hits_refill_kernel<<<static_cast<uint32_t>(grid), 256, smem, c->stream>>>(prm);
  else
    ungapped_kernel<false><<<static_cast<uint32_t>(grid), 256, smem, c->stream>>>(prm);
  ++c->launches;
  ST_CUDA(cudaGetLastError());
  return ST_OK;
}

extern "C" int st_ungapped_score(st_ctx* c, uint32_t profile, const st_lane* lanes, uint32_t n, int32_t* out) {
  CTX_GUARD(c);
  if (n && (!lanes || !out)) return fail(ST_EINVAL, "st_ungapped_score: null argument");
  if (!c->has_db) return fail(ST_ESTATE, "no target database uploaded (st_db_upload)");
  ST_TRY(check_profile(c, profile));
  ST_TRY(sync_profiles(c));
  if (n == 0) return ST_OK;
  const uint32_t m = c->profs[profile].m;
  const size_t jb = up16(static_cast<size_t>(n) * sizeof(UngappedJob));
  ST_TRY(c->pin.reserve(jb + static_cast<size_t>(n) * 4));
  if (c->stage.bytes < jb + static_cast<size_t>(n) * 4) ST_TRY(dev_alloc(&c->mt, c->stage, (jb + n * 4ull) * 2));
  ST_CUDA(cudaStreamSynchronize(c->stream));
  UngappedJob* h = c->pin.as<UngappedJob>();
  for (uint32_t i = 0; i < n; ++i) {
    const st_lane& l = lanes[i];
    if (l.target >= c->n_seqs) return fail(ST_EINVAL, "lane %u: target %u outside the database", i, l.target);
    const int64_t tn = c->h_db_len[l.target];
    // the window must lie inside diag_range (src/ungapped.rs:300-310)
    const int64_t lo = std::max<int64_t>(-static_cast<int64_t>(l.diag), 0);
    const int64_t hi = std::min<int64_t>(m, tn - l.diag);
    UngappedJob j{profile, l.target, l.diag, l.lo, l.hi};
    if (l.lo >= l.hi) {
      j.lo = j.hi = 0;
    } else if (static_cast<int64_t>(l.lo) < lo || static_cast<int64_t>(l.hi) > hi) {
      return fail(ST_EINVAL, "lane %u: window [%u, %u) outside the diagonal's range [%lld, %lld)", i, l.lo, l.hi,
                  static_cast<long long>(lo), static_cast<long long>(hi));
    }
    h[i] = j;
  }
  char* d = c->stage.as<char>();
  ST_CUDA(cudaMemcpyAsync(d, h, static_cast<size_t>(n) * sizeof(UngappedJob), cudaMemcpyHostToDevice, c->stream));
  int32_t* d_out = reinterpret_cast<int32_t*>(d + jb);
  ST_TRY(launch_ungapped(c, false, d, n, d_out, std::max<uint32_t>(m, 1)));
  ST_CUDA(cudaMemcpyAsync(out, d_out, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost, c->stream));
  ST_CUDA(cudaStreamSynchronize(c->stream));
  return ST_OK;
}

// The reference's Lane as it is (src/ungapped.rs:265-270): the target is a
// slice of the database arena that the caller gave st_db_upload (prefilter.rs
// builds lanes from index.seq(tid), src/prefilter.rs:1563-1568).  Each slice is
// mapped back to its sequence by a binary search of the caller's offsets; a
// slice that starts `a` residues into its sequence scores diagonal diag + a of
// the whole sequence over the same query window, which reads the same residues
// (slice[q + diag] = sequence[q + diag + a]).
extern "C" int st_ungapped_score_slices(st_ctx* c, uint32_t profile, const st_lane_slice* lanes, uint32_t n,
                                        int32_t* out) {
  CTX_GUARD(c);
  if (n && (!lanes || !out)) return fail(ST_EINVAL, "st_ungapped_score_slices: null argument");
  if (!c->has_db) return fail(ST_ESTATE, "no target database uploaded (st_db_upload)");
  ST_TRY(check_profile(c, profile));
  if (n == 0) return ST_OK;
  const int64_t m = c->profs[profile].m;
  std::vector<st_lane> mapped(n);
  bool any_live = false;
  const uint64_t* so = c->h_src_off.data();
  const uint64_t first = so[0], last = so[c->n_seqs];
  for (uint32_t i = 0; i < n; ++i) {
    const st_lane_slice& l = lanes[i];
    // diag_range of the slice (src/ungapped.rs:38-46); score_batch requires lo..hi inside it
    const int64_t len = static_cast<int64_t>(l.len);
    const int64_t rlo = std::max<int64_t>(-l.diag, 0);
    const int64_t rhi = std::min<int64_t>(m, len - l.diag);
    if (l.lo >= l.hi || rhi <= rlo) {
      mapped[i] = st_lane{0, 0, 0, 0};  // an empty window scores 0 (kadane_score's best starts at 0)
      continue;
    }
    if (static_cast<int64_t>(l.lo) < rlo || static_cast<int64_t>(l.hi) > rhi)
      return fail(ST_EINVAL, "lane %u: window [%llu, %llu) outside the diagonal's range [%lld, %lld)", i,
                  static_cast<unsigned long long>(l.lo), static_cast<unsigned long long>(l.hi),
                  static_cast<long long>(rlo), static_cast<long long>(rhi));
    const uintptr_t p = reinterpret_cast<uintptr_t>(l.target);
    if (!l.target || p < c->h_src_base || p - c->h_src_base < first || p - c->h_src_base + l.len > last)
      return fail(ST_EINVAL, "lane %u: the target slice is not inside the database arena given to st_db_upload", i);
    const uint64_t pos = p - c->h_src_base;
    // the last sequence starting at or before pos
    const uint64_t* it = std::upper_bound(so, so + c->n_seqs + 1, pos);
    const uint32_t s = static_cast<uint32_t>(it - so - 1);
    if (s >= c->n_seqs || pos + l.len > so[s + 1])
      return fail(ST_EINVAL, "lane %u: the target slice crosses the end of database sequence %u", i, s);
    const int64_t diag = l.diag + static_cast<int64_t>(pos - so[s]);
    if (diag < INT32_MIN || diag > INT32_MAX) return fail(ST_EINVAL, "lane %u: diagonal out of range", i);
    mapped[i] = st_lane{s, static_cast<uint32_t>(l.lo), static_cast<uint32_t>(l.hi), static_cast<int32_t>(diag)};
    any_live = true;
  }
  if (!any_live) {
    std::fill(out, out + n, 0);
    return ST_OK;
  }
  return st_ungapped_score(c, profile, mapped.data(), n, out);
}

// Per-(query, target) runs of hits (consecutive hits with the same query and
// target): one (best, query, target) entry per run, in hit order, by a
// reduce-by-key over the packed (query, target) key. Asynchronous; the
// scratch goes back to the pool behind the stream.
struct HitPairKey {
  __host__ __device__ uint64_t operator()(const HitRec& h) const {
    return (static_cast<uint64_t>(h.query) << 32) | h.target;
  }
};
struct MaxI32 {
  __host__ __device__ int32_t operator()(int32_t a, int32_t b) const { return a > b ? a : b; }
};

__global__ void __launch_bounds__(256) split_pair_keys_kernel(const uint64_t* keys, const uint64_t* n_runs,
                                                              uint32_t* pair_q, uint32_t* pair_t, uint64_t* n_out) {
  const uint64_t n = *n_runs;
  if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = n;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint64_t k = keys[i];
    pair_q[i] = static_cast<uint32_t>(k >> 32);
    pair_t[i] = static_cast<uint32_t>(k);
  }
}

static int run_pairs_device(st_ctx* c, const st_hit* d_hits, uint64_t n, const int32_t* d_per_hit,
                            int32_t* d_pair_best, uint32_t* d_pair_q, uint32_t* d_pair_t, uint64_t* d_n_pairs) {
  const HitRec* h = reinterpret_cast<const HitRec*>(d_hits);
  cub::TransformInputIterator<uint64_t, HitPairKey, const HitRec*> keys(h, HitPairKey());
  size_t t_bytes = 0;
  ST_CUDA(cub::DeviceReduce::ReduceByKey(nullptr, t_bytes, keys, static_cast<uint64_t*>(nullptr), d_per_hit,
                                         d_pair_best, static_cast<uint64_t*>(nullptr), MaxI32(), n, c->stream));
  DevMem tmp;
  const size_t o_keys = 0, o_runs = up256(n * 8), o_cub = o_runs + 256;
  ST_TRY(pool_get(c, o_cub + t_bytes, tmp));
  char* b = tmp.as<char>();
  uint64_t* ukeys = reinterpret_cast<uint64_t*>(b + o_keys);
  uint64_t* runs = reinterpret_cast<uint64_t*>(b + o_runs);
  ST_CUDA(cub::DeviceReduce::ReduceByKey(b + o_cub, t_bytes, keys, ukeys, d_per_hit, d_pair_best, runs, MaxI32(), n,
                                         c->stream));
  const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>((n + 255) / 256, static_cast<uint64_t>(c->sms) * 8));
  split_pair_keys_kernel<<<grid, 256, 0, c->stream>>>(ukeys, runs, d_pair_q, d_pair_t, d_n_pairs);
  ++c->launches;
  ST_CUDA(cudaGetLastError());
  pool_put_after(c, std::move(tmp), c->stream);
  return ST_OK;
}

// Host -> device copy on stream s.  Pinned memory is copied directly; pageable
// memory goes through the two pinned staging blocks in turn (filled by all
// host threads, each uploaded on the copy stream while the next one fills),
// which runs at host memcpy speed instead of the driver's pageable path.
static int upload_host(st_ctx* c, void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return ST_OK;
  if (host_pinned(src)) {
    ST_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    return ST_OK;
  }
  constexpr size_t kChunk = 32ull << 20, kPiece = 1ull << 20;
  if (!c->copy_ev) ST_CUDA(cudaEventCreateWithFlags(&c->copy_ev, cudaEventDisableTiming));
  ST_CUDA(cudaEventRecord(c->copy_ev, s));  // the destination's earlier users come first
  ST_CUDA(cudaStreamWaitEvent(c->copy, c->copy_ev, 0));
  int slot = 0;
  for (size_t o = 0; o < bytes; o += kChunk) {
    const size_t len = std::min(kChunk, bytes - o);
    Pinned& st = c->prof_stage[slot];
    if (!c->prof_stage_ev[slot]) ST_CUDA(cudaEventCreateWithFlags(&c->prof_stage_ev[slot], cudaEventDisableTiming));
    if (c->prof_stage_used[slot]) ST_CUDA(cudaEventSynchronize(c->prof_stage_ev[slot]));
    ST_TRY(st.reserve(kChunk));
    char* h = st.as<char>();
    const char* from = static_cast<const char*>(src) + o;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < static_cast<int64_t>((len + kPiece - 1) / kPiece); ++k)
      memcpy(h + k * kPiece, from + k * kPiece, std::min(kPiece, len - k * kPiece));
    ST_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + o, h, len, cudaMemcpyHostToDevice, c->copy));
    ST_CUDA(cudaEventRecord(c->prof_stage_ev[slot], c->copy));
    c->prof_stage_used[slot] = true;
    slot ^= 1;
  }
  ST_CUDA(cudaEventRecord(c->copy_ev, c->copy));
  ST_CUDA(cudaStreamWaitEvent(s, c->copy_ev, 0));
  return ST_OK;
}

static int check_hits_device(st_ctx* c) {
  if (!c->has_db) return fail(ST_ESTATE, "no target database uploaded (st_db_upload)");
  return sync_profiles(c);
}

extern "C" int st_ungapped_hits_device(st_ctx* c, const st_hit* d_hits, uint64_t n, int32_t* d_per_hit,
                                       int32_t* d_pair_best, uint32_t* d_pair_query, uint32_t* d_pair_target,
                                       uint64_t* d_n_pairs) {
  CTX_GUARD(c);
  if (n && (!d_hits || !d_per_hit)) return fail(ST_EINVAL, "st_ungapped_hits_device: null argument");
  ST_TRY(check_hits_device(c));
  if (n == 0) {
    if (d_n_pairs) ST_CUDA(cudaMemsetAsync(d_n_pairs, 0, 8, c->stream));
    return ST_OK;
  }
  ST_TRY(launch_ungapped(c, true, d_hits, n, d_per_hit));
  if (d_pair_best && d_pair_query && d_pair_target && d_n_pairs)
    ST_TRY(run_pairs_device(c, d_hits, n, d_per_hit, d_pair_best, d_pair_query, d_pair_target, d_n_pairs));
  return ST_OK;
}

extern "C" int st_ungapped_hits(st_ctx* c, const st_hit* hits, uint64_t n, int32_t* per_hit, int32_t* pair_best,
                                uint32_t* pair_query, uint32_t* pair_target, uint64_t* n_pairs) {
  CTX_GUARD(c);
  if (n && (!hits || !per_hit)) return fail(ST_EINVAL, "st_ungapped_hits: null argument");
  ST_TRY(check_hits_device(c));
  const bool want_pairs = pair_best && pair_query && pair_target && n_pairs;
  if (n == 0) {
    if (n_pairs) *n_pairs = 0;
    return ST_OK;
  }
  uint32_t max_m = 1;
  for (uint64_t i = 0; i < n; ++i) {
    if (hits[i].query >= c->profs.size() || !c->profs[hits[i].query].live)
      return fail(ST_EINVAL, "hit %llu: unknown profile id %u", static_cast<unsigned long long>(i), hits[i].query);
    if (hits[i].target >= c->n_seqs)
      return fail(ST_EINVAL, "hit %llu: target %u outside the database", static_cast<unsigned long long>(i),
                  hits[i].target);
    max_m = std::max(max_m, c->profs[hits[i].query].m);
  }
  DevMem buf;
  const size_t hb = up16(n * sizeof(st_hit));
  const size_t ob = up16(n * 4);
  ST_TRY(pool_get(c, hb + ob + (want_pairs ? 3 * ob + 16 : 0), buf));
  struct Back {
    st_ctx* c;
    DevMem* m;
    ~Back() { pool_put_after(c, std::move(*m), c->stream); }
  } back{c, &buf};
  char* d = buf.as<char>();
  ST_TRY(upload_host(c, d, hits, n * sizeof(st_hit), c->stream));
  int32_t* d_out = reinterpret_cast<int32_t*>(d + hb);
  ST_TRY(launch_ungapped(c, true, d, n, d_out, max_m));
  if (want_pairs) {
    int32_t* d_pb = reinterpret_cast<int32_t*>(d + hb + ob);
    uint32_t* d_pq = reinterpret_cast<uint32_t*>(d + hb + 2 * ob);
    uint32_t* d_pt = reinterpret_cast<uint32_t*>(d + hb + 3 * ob);
    uint64_t* d_np = reinterpret_cast<uint64_t*>(d + hb + 4 * ob);
    ST_TRY(run_pairs_device(c, reinterpret_cast<const st_hit*>(d), n, d_out, d_pb, d_pq, d_pt, d_np));
    uint64_t np = 0;
    ST_CUDA(cudaMemcpyAsync(&np, d_np, 8, cudaMemcpyDeviceToHost, c->stream));
    ST_CUDA(cudaStreamSynchronize(c->stream));
    *n_pairs = np;
    if (np) {
      ST_CUDA(cudaMemcpyAsync(pair_best, d_pb, np * 4, cudaMemcpyDeviceToHost, c->stream));
      ST_CUDA(cudaMemcpyAsync(pair_query, d_pq, np * 4, cudaMemcpyDeviceToHost, c->stream));
      ST_CUDA(cudaMemcpyAsync(pair_target, d_pt, np * 4, cudaMemcpyDeviceToHost, c->stream));
    }
  }
  ST_CUDA(cudaMemcpyAsync(per_hit, d_out, n * 4, cudaMemcpyDeviceToHost, c->stream));
  ST_CUDA(cudaStreamSynchronize(c->stream));
  return ST_OK;
}

// ---------------------------------------------------------------------------
// prefilter evidence, chain and gate (st_gate.cuh)
// ---------------------------------------------------------------------------
static_assert(sizeof(st_seed_hit) == sizeof(GateSeedHit), "seed hit layout");
static_assert(sizeof(st_candidate) == sizeof(GateCandidate), "candidate layout");
static_assert(sizeof(st_prefilter_stats) == sizeof(GateStats), "stats layout");

static int gate_conf(st_ctx* c, const st_prefilter_params* p, GateConf& g, int& qbits) {
  if (!p) return fail(ST_EINVAL, "null prefilter parameters");
  if (p->max_diagonals == 0) return fail(ST_EINVAL, "max_diagonals must be at least 1");
  if (p->diag_hits == 0) return fail(ST_EINVAL, "diag_hits must be at least 1");
  if (!c->has_db) return fail(ST_ESTATE, "no target database uploaded (st_db_upload)");
  ST_TRY(sync_profiles(c));
  g.min_hits = p->min_hits;
  g.diag_hits = p->diag_hits;
  g.kmax = std::min<uint32_t>(p->max_diagonals, kGateMaxDiags);
  g.window = p->diag_window;
  g.span = p->span;
  g.min_score = p->min_diag_score;
  g.open = p->gap_open;
  g.ext = p->gap_ext;
  g.max_cand = p->max_candidates;
  g.regions = p->regions ? 1u : 0u;
  g.n_prof = static_cast<uint32_t>(c->profs.size());
  g.tbits = static_cast<uint32_t>(bits_for(c->n_seqs ? c->n_seqs - 1 : 0));
  g.doff = c->max_m;
  g.dbits = static_cast<uint32_t>(bits_for(static_cast<uint64_t>(c->max_m) + c->max_len));
  qbits = bits_for(g.n_prof);  // n_prof itself marks rejected hits
  if (qbits + static_cast<int>(g.tbits + g.dbits) > 64 || qbits > 32)
    return fail(ST_EINVAL, "seed-hit key needs %d bits (query %d, target %u, diagonal %u); at most 64",
                qbits + static_cast<int>(g.tbits + g.dbits), qbits, g.tbits, g.dbits);
  g.stride = ung_stride(c);
  if (16 + static_cast<size_t>(kProfRows) * g.stride + 16 > static_cast<size_t>(g_gate_smem))
    return fail(ST_EINVAL, "query too long for the prefilter segment kernel (%u rows)", c->max_m);
  return ST_OK;
}

// The whole pipeline on the context stream, one host synchronisation (the
// number of candidates, which sizes the ranking sort) and a final one for the
// counts.  Ranked candidates go to d_out (room for n entries).
static int gate_pipeline(st_ctx* c, const GateSeedHit* d_hits, uint32_t n, const GateConf& g, int qbits,
                         GateCandidate* d_out, uint64_t* n_out, GateStats* h_stats) {
  const int key_bits = qbits + static_cast<int>(g.tbits + g.dbits);
  const size_t P = static_cast<size_t>(g.n_prof) + 1;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t r = o;
    o += up256(std::max<size_t>(bytes, 1));
    return r;
  };
  const size_t o_k0 = take(8ull * n), o_k1 = take(8ull * n), o_v0 = take(4ull * n), o_v1 = take(4ull * n);
  const size_t o_start = take(4ull * n), o_ng = take(4), o_ns = take(4ull * (n + 1)), o_joff = take(4ull * (n + 1));
  const size_t o_jobs = take(sizeof(GateJob) * n), o_sc = take(4ull * n);
  const size_t o_cand = take(sizeof(GateCandidate) * n), o_flag = take(n), o_sel = take(4ull * n), o_nc = take(4);
  const size_t o_work = take(4ull * n), o_nw = take(4);
  const size_t o_stats = take(sizeof(GateStats)), o_nout = take(8);
  const size_t o_qf = take(4 * P), o_qend = take(4 * P), o_kept = take(4 * P), o_koff = take(4 * P);
  // CUB scratch, sized for the largest input of each call
  size_t t_max = 0, t = 0;
  {
    cub::DoubleBuffer<uint64_t> kb(nullptr, nullptr);
    cub::DoubleBuffer<uint32_t> vb(nullptr, nullptr);
    ST_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t, kb, vb, n, 0, key_bits, c->stream));
    t_max = std::max(t_max, t);
    ST_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t, kb, vb, n, 0, 31 + qbits, c->stream));
    t_max = std::max(t_max, t);
    cub::CountingInputIterator<uint32_t> it(0);
    ST_CUDA(cub::DeviceSelect::Flagged(nullptr, t, it, static_cast<const uint8_t*>(nullptr),
                                       static_cast<uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr), n,
                                       c->stream));
    t_max = std::max(t_max, t);
    ST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t, static_cast<uint32_t*>(nullptr),
                                          static_cast<uint32_t*>(nullptr), n + 1, c->stream));
    t_max = std::max(t_max, t);
    ST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t, static_cast<uint32_t*>(nullptr),
                                          static_cast<uint32_t*>(nullptr), P, c->stream));
    t_max = std::max(t_max, t);
  }
  const size_t o_tmp = take(t_max);
  TraceClock tc("gate");
  DevMem mem;
  ST_TRY(pool_get(c, o, mem));
  tc.lap("scratch");
  struct Back {
    st_ctx* c;
    DevMem* m;
    ~Back() { pool_put_after(c, std::move(*m), c->stream); }
  } back{c, &mem};
  char* b = mem.as<char>();
  auto at = [&](size_t off) { return static_cast<void*>(b + off); };
  uint64_t* k0 = static_cast<uint64_t*>(at(o_k0));
  uint64_t* k1 = static_cast<uint64_t*>(at(o_k1));
  uint32_t* v0 = static_cast<uint32_t*>(at(o_v0));
  uint32_t* v1 = static_cast<uint32_t*>(at(o_v1));
  uint32_t* start = static_cast<uint32_t*>(at(o_start));
  uint32_t* ng = static_cast<uint32_t*>(at(o_ng));
  uint32_t* ns = static_cast<uint32_t*>(at(o_ns));
  uint32_t* joff = static_cast<uint32_t*>(at(o_joff));
  GateJob* jobs = static_cast<GateJob*>(at(o_jobs));
  int32_t* sc = static_cast<int32_t*>(at(o_sc));
  GateCandidate* cand = static_cast<GateCandidate*>(at(o_cand));
  uint8_t* flag = static_cast<uint8_t*>(at(o_flag));
  uint32_t* sel = static_cast<uint32_t*>(at(o_sel));
  uint32_t* nc = static_cast<uint32_t*>(at(o_nc));
  uint32_t* work = static_cast<uint32_t*>(at(o_work));
  uint32_t* n_work = static_cast<uint32_t*>(at(o_nw));
  GateStats* st = static_cast<GateStats*>(at(o_stats));
  unsigned long long* nout = static_cast<unsigned long long*>(at(o_nout));
  uint32_t* qf = static_cast<uint32_t*>(at(o_qf));
  uint32_t* qend = static_cast<uint32_t*>(at(o_qend));
  uint32_t* kept = static_cast<uint32_t*>(at(o_kept));
  uint32_t* koff = static_cast<uint32_t*>(at(o_koff));
  void* tmp = at(o_tmp);
  cudaStream_t s = c->stream;
  // enough blocks for every SM to hold its full 2048 threads several times over
  auto grid_for = [&](uint64_t items, uint32_t block) {
    const uint64_t cap = static_cast<uint64_t>(c->sms) * (2048 / block) * 4;
    return static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>((items + block - 1) / block, cap)));
  };
  ST_CUDA(cudaMemsetAsync(st, 0, sizeof(GateStats), s));
  // keys, sort, groups
  DeviceDb db = db_view(c);
  DeviceProfiles pv = prof_view(c);
  gate_keys_kernel<<<grid_for(n, 256), 256, 0, s>>>(d_hits, n, db, pv.qlen, g, k0, v0, st);
  cub::DoubleBuffer<uint64_t> kb(k0, k1);
  cub::DoubleBuffer<uint32_t> vb(v0, v1);
  t = t_max;
  ST_CUDA(cub::DeviceRadixSort::SortPairs(tmp, t, kb, vb, n, 0, key_bits, s));
  GateGroups G{kb.Current(), vb.Current(), start, ng, n};
  {
    cub::CountingInputIterator<uint32_t> it(0);
    cub::TransformInputIterator<bool, GateHeadFlag, cub::CountingInputIterator<uint32_t>> heads(
        it, GateHeadFlag{kb.Current(), g.dbits});
    t = t_max;
    ST_CUDA(cub::DeviceSelect::Flagged(tmp, t, it, heads, start, ng, n, s));
  }
  // jobs
  gate_count_kernel<<<grid_for(static_cast<uint64_t>(n) + 1, 256), 256, 0, s>>>(G, g, ns, st);
  t = t_max;
  ST_CUDA(cub::DeviceScan::ExclusiveSum(tmp, t, ns, joff, n + 1, s));
  if (g.kmax <= 4)
    gate_emit_kernel<4><<<grid_for(n, 128), 128, 0, s>>>(G, g, db, pv.qlen, ns, joff, jobs);
  else
    gate_emit_kernel<kGateMaxDiags><<<grid_for(n, 128), 128, 0, s>>>(G, g, db, pv.qlen, ns, joff, jobs);
  // window scores
  GateSegParams sp{db, pv, jobs, ng, joff, sc, g.stride};
  const size_t smem = 16 + static_cast<size_t>(kProfRows) * sp.max_m_pad + 16;
  gate_score_kernel<<<static_cast<uint32_t>((static_cast<uint64_t>(n) + kGateChunk - 1) / kGateChunk), 256, smem, s>>>(
      sp);
  // chain, gate, compaction
  ST_CUDA(cudaMemsetAsync(flag, 0, n, s));
  ST_CUDA(cudaMemsetAsync(n_work, 0, 4, s));
  gate_screen_kernel<<<grid_for(n, 256), 256, 0, s>>>(G, g, joff, sc, work, n_work);
  gate_chain_kernel<<<grid_for(n, 128), 128, 0, s>>>(G, g, db, pv, joff, jobs, sc, work, n_work, cand, flag, st);
  {
    cub::CountingInputIterator<uint32_t> it(0);
    t = t_max;
    ST_CUDA(cub::DeviceSelect::Flagged(tmp, t, it, flag, sel, nc, n, s));
  }
  c->launches += 8;
  ST_CUDA(cudaGetLastError());
  ST_TRY(c->pin.reserve(64));
  uint32_t* h_nc = c->pin.as<uint32_t>();
  tc.lap("enqueue");
  ST_CUDA(cudaMemcpyAsync(h_nc, nc, 4, cudaMemcpyDeviceToHost, s));
  ST_CUDA(cudaStreamSynchronize(s));
  const uint32_t n_cand = *h_nc;
  tc.lap("device");
  // ranking: the sort keys reuse the hit-key buffers (free after the jobs are emitted)
  if (n_cand) {
    gate_rank_keys_kernel<<<grid_for(n_cand, 256), 256, 0, s>>>(cand, sel, nc, k0, v0);
    cub::DoubleBuffer<uint64_t> rk(k0, k1);
    cub::DoubleBuffer<uint32_t> ri(v0, v1);
    t = t_max;
    ST_CUDA(cub::DeviceRadixSort::SortPairs(tmp, t, rk, ri, n_cand, 0, 31 + qbits, s));
    if (g.max_cand) {
      ST_CUDA(cudaMemsetAsync(qf, 0, 4 * P, s));
      ST_CUDA(cudaMemsetAsync(qend, 0, 4 * P, s));
      gate_query_bounds_kernel<<<grid_for(n_cand, 256), 256, 0, s>>>(rk.Current(), nc, qf, qend);
      gate_query_kept_kernel<<<grid_for(P, 256), 256, 0, s>>>(qf, qend, g.n_prof, g.max_cand, kept);
      t = t_max;
      ST_CUDA(cub::DeviceScan::ExclusiveSum(tmp, t, kept, koff, P, s));
      c->launches += 2;
    }
    gate_gather_kernel<<<grid_for(n_cand, 256), 256, 0, s>>>(cand, rk.Current(), ri.Current(), nc, g.max_cand, qf,
                                                             koff, d_out);
    c->launches += 2;
  }
  gate_finish_kernel<<<1, 1, 0, s>>>(ng, joff, nc, koff, g.n_prof, n_cand ? g.max_cand : 0, st, nout);
  ++c->launches;
  ST_CUDA(cudaGetLastError());
  GateStats* h_st = reinterpret_cast<GateStats*>(c->pin.as<char>());
  ST_CUDA(cudaMemcpyAsync(h_st, st, sizeof(GateStats), cudaMemcpyDeviceToHost, s));
  ST_CUDA(cudaStreamSynchronize(s));
  *h_stats = *h_st;
  *n_out = h_st->candidates;
  tc.lap("rank (enqueue + device)");
  return ST_OK;
}

static int gate_check_n(uint64_t n) {
  if (n >= 0x7FFFFFFFull) return fail(ST_EINVAL, "too many seed hits in one call (%llu; fewer than 2^31 - 1)",
                                      static_cast<unsigned long long>(n));
  return ST_OK;
}

static int gate_result(const GateStats& st, st_prefilter_stats* stats) {
  if (stats) memcpy(stats, &st, sizeof st);
  if (st.hits_rejected)
    return fail(ST_EINVAL, "%llu seed hits lie outside their query or target (unknown ids or positions)",
                st.hits_rejected);
  return ST_OK;
}

extern "C" int st_prefilter_gate_device(st_ctx* c, const st_seed_hit* d_hits, uint64_t n,
                                        const st_prefilter_params* params, st_candidate* d_out, uint64_t* n_out,
                                        st_prefilter_stats* stats) {
  CTX_GUARD(c);
  if (!n_out || (n && (!d_hits || !d_out))) return fail(ST_EINVAL, "st_prefilter_gate_device: null argument");
  ST_TRY(gate_check_n(n));
  GateConf g;
  int qbits = 0;
  ST_TRY(gate_conf(c, params, g, qbits));
  GateStats st{};
  *n_out = 0;
  if (n)
    ST_TRY(gate_pipeline(c, reinterpret_cast<const GateSeedHit*>(d_hits), static_cast<uint32_t>(n), g, qbits,
                         reinterpret_cast<GateCandidate*>(d_out), n_out, &st));
  return gate_result(st, stats);
}

extern "C" int st_prefilter_gate(st_ctx* c, const st_seed_hit* hits, uint64_t n, const st_prefilter_params* params,
                                 st_candidate* out, uint64_t cap, uint64_t* n_out, st_prefilter_stats* stats) {
  CTX_GUARD(c);
  if (!n_out || (n && !hits) || (cap && !out)) return fail(ST_EINVAL, "st_prefilter_gate: null argument");
  ST_TRY(gate_check_n(n));
  GateConf g;
  int qbits = 0;
  ST_TRY(gate_conf(c, params, g, qbits));
  GateStats st{};
  *n_out = 0;
  if (n) {
    DevMem buf;
    const size_t hb = up256(n * sizeof(st_seed_hit));
    ST_TRY(pool_get(c, hb + n * sizeof(st_candidate), buf));
    struct Back {
      st_ctx* c;
      DevMem* m;
      ~Back() { pool_put_after(c, std::move(*m), c->stream); }
    } back{c, &buf};
    char* d = buf.as<char>();
    ST_TRY(upload_host(c, d, hits, n * sizeof(st_seed_hit), c->stream));
    GateCandidate* d_out = reinterpret_cast<GateCandidate*>(d + hb);
    ST_TRY(gate_pipeline(c, reinterpret_cast<const GateSeedHit*>(d), static_cast<uint32_t>(n), g, qbits, d_out,
                         n_out, &st));
    const uint64_t k = std::min<uint64_t>(cap, *n_out);
    if (k) {
      ST_CUDA(cudaMemcpyAsync(out, d_out, k * sizeof(st_candidate), cudaMemcpyDeviceToHost, c->stream));
      ST_CUDA(cudaStreamSynchronize(c->stream));
    }
  }
  return gate_result(st, stats);
}

// ---------------------------------------------------------------------------
// seed index and seed hits (st_seed.cuh)
// ---------------------------------------------------------------------------
static_assert(sizeof(st_seed_stats) == 9 * 8, "seed stats layout");

extern "C" int st_seed_index_build(st_ctx* c, const char* mask) {
  CTX_GUARD(c);
  if (!mask) return fail(ST_EINVAL, "st_seed_index_build: null seed mask");
  if (!c->has_db) return fail(ST_ESTATE, "no target database uploaded (st_db_upload)");
  // SeedPattern::from_mask (src/prefilter.rs:101-124)
  SeedPat p{};
  const size_t len = strlen(mask);
  for (size_t i = 0; i < len; ++i) {
    if (mask[i] != '0' && mask[i] != '1') return fail(ST_EINVAL, "seed mask must be 0/1, got '%c'", mask[i]);
    if (mask[i] == '1') {
      if (p.w >= static_cast<uint32_t>(kSeedMaxW))
        return fail(ST_EINVAL, "seed weight above %d is not supported by the device index", kSeedMaxW);
      p.offs[p.w++] = static_cast<uint32_t>(i);
    }
  }
  if (len == 0 || p.w == 0) return fail(ST_EINVAL, "seed mask has no care ('1') positions");
  if (mask[0] != '1' || mask[len - 1] != '1') return fail(ST_EINVAL, "seed mask must start and end with '1'");
  if (p.w < 2) return fail(ST_EINVAL, "seed weight below 2 is not supported");
  p.span = static_cast<uint32_t>(len);
  uint64_t n_codes = 1;
  for (uint32_t i = 0; i < p.w; ++i) n_codes *= kSeedAA;
  c->has_seed_index = false;
  ST_TRY(dev_alloc(&c->mt, c->seed_off, (n_codes + 1) * 4));
  size_t t_scan = 0;
  ST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t_scan, static_cast<uint32_t*>(nullptr),
                                        static_cast<uint32_t*>(nullptr), n_codes + 1, c->stream));
  DevMem tmp;
  ST_TRY(pool_get(c, up256((n_codes + 1) * 4) + t_scan, tmp));
  uint32_t* cnt = tmp.as<uint32_t>();
  void* cub_tmp = tmp.as<char>() + up256((n_codes + 1) * 4);
  ST_CUDA(cudaMemsetAsync(cnt, 0, (n_codes + 1) * 4, c->stream));
  const DeviceDb db = db_view(c);
  const uint32_t blocks = static_cast<uint32_t>(
      std::max<uint64_t>(1, std::min<uint64_t>((c->n_seqs + 7) / 8, static_cast<uint64_t>(c->sms) * 32)));
  seed_index_kernel<false><<<blocks, 256, 0, c->stream>>>(db, p, cnt, nullptr);
  ST_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp, t_scan, cnt, c->seed_off.as<uint32_t>(), n_codes + 1, c->stream));
  // postings: the scan's last entry, read back once
  ST_TRY(c->pin.reserve(64));
  uint32_t* h_total = c->pin.as<uint32_t>();
  ST_CUDA(cudaMemcpyAsync(h_total, c->seed_off.as<uint32_t>() + n_codes, 4, cudaMemcpyDeviceToHost, c->stream));
  ST_CUDA(cudaStreamSynchronize(c->stream));
  const uint64_t n_post = *h_total;
  // every window of the database is counted at most once; 32-bit offsets hold it below 2^32
  if (c->n_res >= 0xFFFFFFFFull) return fail(ST_EINVAL, "database too large for 32-bit seed-index offsets");
  ST_TRY(dev_alloc(&c->mt, c->seed_post, std::max<uint64_t>(n_post, 1) * sizeof(SeedPost)));
  ST_CUDA(cudaMemcpyAsync(cnt, c->seed_off.p, n_codes * 4, cudaMemcpyDeviceToDevice, c->stream));
  seed_index_kernel<true><<<blocks, 256, 0, c->stream>>>(db, p, cnt, c->seed_post.as<SeedPost>());
  c->launches += 4;
  ST_CUDA(cudaGetLastError());
  ST_CUDA(cudaStreamSynchronize(c->stream));
  pool_put(c, std::move(tmp));
  c->seed_pat = p;
  c->seed_n_post = n_post;
  c->has_seed_index = true;
  return ST_OK;
}

// The seed stage for a batch of queries: hits (device, pooled in `hits`), their
// count and the counters.  Two host synchronisations (seed slots, hits) size
// the buffers.
static int seed_stage(st_ctx* c, const uint32_t* profiles, uint32_t n_q, const uint8_t* residues,
                      const uint64_t* res_off, const st_seed_params* sp, DevMem& hits, uint32_t* n_hits,
                      st_seed_stats* stats) {
  if (!sp) return fail(ST_EINVAL, "null seed parameters");
  if (sp->max_kmers_per_pos == 0) return fail(ST_EINVAL, "max_kmers_per_pos must be at least 1");
  if (!c->has_db) return fail(ST_ESTATE, "no target database uploaded (st_db_upload)");
  if (!c->has_seed_index) return fail(ST_ESTATE, "no seed index for the current database (st_seed_index_build)");
  if (n_q && !profiles) return fail(ST_EINVAL, "null profile ids");
  if (residues && !res_off) return fail(ST_EINVAL, "residues without offsets");
  const SeedPat& P = c->seed_pat;
  std::vector<uint32_t> woff(static_cast<size_t>(n_q) + 1), row0(static_cast<size_t>(n_q) + 1);
  uint64_t nw = 0, nr = 0;
  for (uint32_t i = 0; i < n_q; ++i) {
    ST_TRY(check_profile(c, profiles[i]));
    const uint64_t m = c->profs[profiles[i]].m;
    if (residues && res_off[i + 1] - res_off[i] != m)
      return fail(ST_EINVAL, "query %u: %llu residues for a profile of %llu rows", i,
                  static_cast<unsigned long long>(res_off[i + 1] - res_off[i]), static_cast<unsigned long long>(m));
    woff[i] = static_cast<uint32_t>(nw);
    row0[i] = static_cast<uint32_t>(nr);
    nw += m >= P.span ? m - P.span + 1 : 0;
    nr += m;
    if (nw >= 0x7FFFFFFFull || nr >= 0x7FFFFFFFull) return fail(ST_EINVAL, "too many query positions in one call");
  }
  woff[n_q] = static_cast<uint32_t>(nw);
  row0[n_q] = static_cast<uint32_t>(nr);
  memset(stats, 0, sizeof *stats);
  stats->windows = nw;
  *n_hits = 0;
  if (nw == 0) return ST_OK;
  TraceClock tc("seeds");
  ST_TRY(sync_profiles(c));
  cudaStream_t s = c->stream;
  // windows: sorted rows, counts, slots
  size_t t_scan = 0;
  ST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t_scan, static_cast<uint32_t*>(nullptr),
                                        static_cast<uint32_t*>(nullptr), nw + 1, s));
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t r = o;
    o += up256(std::max<size_t>(bytes, 1));
    return r;
  };
  const size_t o_q = take(4ull * n_q), o_wo = take(4ull * (n_q + 1)), o_r0 = take(4ull * (n_q + 1));
  const size_t o_res = take(residues ? nr : 0), o_rows = take(sizeof(SeedRow) * nr);
  const size_t o_slots = take(4 * (nw + 1)), o_soff = take(4 * (nw + 1)), o_win = take(sizeof(SeedWin) * nw);
  const size_t o_st = take(sizeof(SeedStatsDev)), o_tmp = take(t_scan);
  tc.lap("windows (prep)");
  DevMem wm;
  ST_TRY(pool_get(c, o, wm));
  tc.lap("windows (scratch)");
  struct Back {
    st_ctx* c;
    DevMem* m;
    ~Back() { pool_put_after(c, std::move(*m), c->stream); }
  } back_w{c, &wm};
  char* b = wm.as<char>();
  ST_CUDA(cudaMemcpyAsync(b + o_q, profiles, 4ull * n_q, cudaMemcpyHostToDevice, s));
  ST_CUDA(cudaMemcpyAsync(b + o_wo, woff.data(), 4ull * (n_q + 1), cudaMemcpyHostToDevice, s));
  ST_CUDA(cudaMemcpyAsync(b + o_r0, row0.data(), 4ull * (n_q + 1), cudaMemcpyHostToDevice, s));
  if (residues) ST_TRY(upload_host(c, b + o_res, residues + res_off[0], nr, s));
  tc.lap("windows (uploads)");
  SeedStatsDev* st = reinterpret_cast<SeedStatsDev*>(b + o_st);
  ST_CUDA(cudaMemsetAsync(st, 0, sizeof(SeedStatsDev), s));
  SeedQ Q;
  Q.qids = reinterpret_cast<const uint32_t*>(b + o_q);
  Q.woff = reinterpret_cast<const uint32_t*>(b + o_wo);
  Q.row0 = reinterpret_cast<const uint32_t*>(b + o_r0);
  Q.res = residues ? reinterpret_cast<const uint8_t*>(b + o_res) : nullptr;
  Q.rows = reinterpret_cast<const SeedRow*>(b + o_rows);
  Q.n_q = n_q;
  Q.n_win = static_cast<uint32_t>(nw);
  Q.thr = sp->kmer_score;
  Q.cap = sp->max_kmers_per_pos;
  Q.exact = (residues && sp->exact_seeds) ? 1u : 0u;
  uint32_t* slots = reinterpret_cast<uint32_t*>(b + o_slots);
  uint32_t* soff = reinterpret_cast<uint32_t*>(b + o_soff);
  SeedWin* win = reinterpret_cast<SeedWin*>(b + o_win);
  auto grid_for = [&](uint64_t items, uint32_t block) {
    const uint64_t cap = static_cast<uint64_t>(c->sms) * (2048 / block) * 4;
    return static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>((items + block - 1) / block, cap)));
  };
  seed_sort_rows_kernel<<<n_q, 128, 0, s>>>(prof_view(c), Q.qids, Q.row0, const_cast<SeedRow*>(Q.rows));
  seed_count_kernel<<<grid_for(nw + 1, 128), 128, 0, s>>>(Q, P, slots, win, st);
  size_t t = t_scan;
  ST_CUDA(cub::DeviceScan::ExclusiveSum(b + o_tmp, t, slots, soff, nw + 1, s));
  c->launches += 3;
  ST_CUDA(cudaGetLastError());
  ST_TRY(c->pin.reserve(64));
  uint32_t* h = c->pin.as<uint32_t>();
  tc.lap("windows (enqueue)");
  ST_CUDA(cudaMemcpyAsync(h, soff + nw, 4, cudaMemcpyDeviceToHost, s));
  ST_CUDA(cudaStreamSynchronize(s));
  const uint64_t ns = *h;
  tc.lap("windows (device)");
  // seeds: k-mers, posting counts, hit offsets
  size_t t_scan2 = 0;
  ST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t_scan2, static_cast<uint32_t*>(nullptr),
                                        static_cast<uint32_t*>(nullptr), ns + 1, s));
  o = 0;
  const size_t o_seeds = take(sizeof(SeedSeed) * ns), o_cnt = take(4 * (ns + 1)), o_hoff = take(4 * (ns + 1));
  const size_t o_tmp2 = take(t_scan2);
  DevMem sm;
  ST_TRY(pool_get(c, o, sm));
  struct Back back_s{c, &sm};
  char* b2 = sm.as<char>();
  SeedSeed* seeds = reinterpret_cast<SeedSeed*>(b2 + o_seeds);
  uint32_t* cnt = reinterpret_cast<uint32_t*>(b2 + o_cnt);
  uint32_t* hoff = reinterpret_cast<uint32_t*>(b2 + o_hoff);
  if (ns) seed_emit_kernel<<<grid_for(nw, 128), 128, 0, s>>>(Q, P, soff, win, seeds, st);
  seed_post_count_kernel<<<grid_for(ns + 1, 256), 256, 0, s>>>(seeds, static_cast<uint32_t>(ns),
                                                               c->seed_off.as<uint32_t>(),
                                                               sp->max_seed_occ, cnt, st);
  t = t_scan2;
  ST_CUDA(cub::DeviceScan::ExclusiveSum(b2 + o_tmp2, t, cnt, hoff, ns + 1, s));
  c->launches += 3;
  ST_CUDA(cudaGetLastError());
  ST_TRY(c->pin.reserve(sizeof(SeedStatsDev) + 64));
  SeedStatsDev* hst = reinterpret_cast<SeedStatsDev*>(c->pin.as<char>());
  uint32_t* h_hits = reinterpret_cast<uint32_t*>(c->pin.as<char>() + sizeof(SeedStatsDev));
  ST_CUDA(cudaMemcpyAsync(hst, st, sizeof(SeedStatsDev), cudaMemcpyDeviceToHost, s));
  tc.lap("k-mers (enqueue)");
  ST_CUDA(cudaMemcpyAsync(h_hits, hoff + ns, 4, cudaMemcpyDeviceToHost, s));
  ST_CUDA(cudaStreamSynchronize(s));
  tc.lap("k-mers (device)");
  const SeedStatsDev sd = *hst;
  const uint64_t nh = *h_hits;
  stats->windows_skipped = sd.windows_skipped;
  stats->kmers_generated = sd.kmers_generated;
  stats->windows_at_cap = sd.windows_at_cap;
  stats->exact_seeds_added = sd.exact_seeds_added;
  stats->seeds = sd.seeds;
  stats->postings_visited = sd.postings_visited;
  stats->seeds_over_occ_cap = sd.seeds_over_occ_cap;
  stats->postings_skipped_occ = sd.postings_skipped_occ;
  if (sd.errors)
    return fail(ST_EINVAL, "%llu windows have a score range above %d histogram bins (rows too wide for the "
                "device seed generator)", sd.errors, kSeedMaxBins);
  if (sd.postings_visited >= 0x7FFFFFFFull) return fail(ST_EINVAL, "too many seed hits in one call");
  ST_TRY(pool_get(c, std::max<uint64_t>(nh, 1) * sizeof(GateSeedHit), hits));
  if (nh) {
    seed_hits_kernel<<<grid_for(ns, 256), 256, 0, s>>>(Q, seeds, static_cast<uint32_t>(ns), cnt, hoff,
                                                       c->seed_off.as<uint32_t>(), c->seed_post.as<SeedPost>(),
                                                       hits.as<GateSeedHit>());
    ++c->launches;
    ST_CUDA(cudaGetLastError());
  }
  *n_hits = static_cast<uint32_t>(nh);
  tc.lap("hits (enqueue)");
  return ST_OK;
}

extern "C" int st_seed_hits(st_ctx* c, const uint32_t* profiles, uint32_t n_queries, const uint8_t* residues,
                            const uint64_t* residue_offsets, const st_seed_params* params, st_seed_hit* out,
                            uint64_t cap, uint64_t* n_out, st_seed_stats* stats) {
  CTX_GUARD(c);
  if (!n_out || (cap && !out)) return fail(ST_EINVAL, "st_seed_hits: null argument");
  DevMem hits;
  uint32_t nh = 0;
  st_seed_stats st{};
  *n_out = 0;
  ST_TRY(seed_stage(c, profiles, n_queries, residues, residue_offsets, params, hits, &nh, &st));
  if (stats) *stats = st;
  *n_out = nh;
  const uint64_t k = std::min<uint64_t>(cap, nh);
  if (k) ST_CUDA(cudaMemcpyAsync(out, hits.p, k * sizeof(st_seed_hit), cudaMemcpyDeviceToHost, c->stream));
  ST_CUDA(cudaStreamSynchronize(c->stream));
  pool_put(c, std::move(hits));
  return ST_OK;
}

// Queries are taken in chunks of at most this many seed windows (about 250
// queries of 250 residues), which bounds the hits held on the device at once.
constexpr uint64_t kSearchChunkWindows = 1ull << 16;

extern "C" int st_prefilter_queries(st_ctx* c, const uint32_t* profiles, uint32_t n_queries, const uint8_t* residues,
                                    const uint64_t* residue_offsets, const st_seed_params* seed_params,
                                    const st_prefilter_params* params, st_candidate* out, uint64_t cap,
                                    uint64_t* n_out, st_prefilter_stats* stats, st_seed_stats* seed_stats) {
  CTX_GUARD(c);
  if (!n_out || (cap && !out) || !params || (n_queries && !profiles))
    return fail(ST_EINVAL, "st_prefilter_queries: null argument");
  if (residues && !residue_offsets) return fail(ST_EINVAL, "residues without offsets");
  *n_out = 0;
  if (!c->has_seed_index) return fail(ST_ESTATE, "no seed index for the current database (st_seed_index_build)");
  st_prefilter_params gp = *params;
  gp.span = c->seed_pat.span;  // the index's seed pattern sets the window span
  GateConf g;
  int qbits = 0;
  ST_TRY(gate_conf(c, &gp, g, qbits));
  std::vector<uint8_t> seen(c->profs.size(), 0);
  for (uint32_t i = 0; i < n_queries; ++i) {
    ST_TRY(check_profile(c, profiles[i]));
    if (seen[profiles[i]]++)  // the evidence stage groups hits by profile id
      return fail(ST_EINVAL, "profile id %u appears twice in one call", profiles[i]);
    if (residues && (residue_offsets[i + 1] < residue_offsets[i] ||
                     residue_offsets[i + 1] - residue_offsets[i] != c->profs[profiles[i]].m))
      return fail(ST_EINVAL, "query %u: residue count differs from its profile's rows", i);
  }
  GateStats tot{};
  st_seed_stats stot{};
  std::vector<st_candidate> all;
  // queries in order of length, so that a chunk's staged profile rows (sized by its longest query) stay short
  std::vector<uint32_t> order(n_queries);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    return c->profs[profiles[a]].m < c->profs[profiles[b]].m;
  });
  uint32_t q0 = 0;
  while (q0 < n_queries) {
    uint32_t q1 = q0;
    uint64_t wins = 0;
    uint32_t max_m = 0;
    std::vector<uint32_t> cp;
    std::vector<uint8_t> cres;
    std::vector<uint64_t> coff(1, 0);
    do {
      const uint32_t qi = order[q1];
      const uint64_t m = c->profs[profiles[qi]].m;
      wins += m >= c->seed_pat.span ? m - c->seed_pat.span + 1 : 0;
      max_m = std::max<uint32_t>(max_m, static_cast<uint32_t>(m));
      cp.push_back(profiles[qi]);
      if (residues) {
        cres.insert(cres.end(), residues + residue_offsets[qi], residues + residue_offsets[qi + 1]);
        coff.push_back(cres.size());
      }
      ++q1;
    } while (q1 < n_queries && wins < kSearchChunkWindows);
    GateConf gc = g;
    gc.stride = static_cast<uint32_t>(up16(max_m) + 32);
    DevMem hits;
    uint32_t nh = 0;
    st_seed_stats sst{};
    ST_TRY(seed_stage(c, cp.data(), q1 - q0, residues ? cres.data() : nullptr, residues ? coff.data() : nullptr,
                      seed_params, hits, &nh, &sst));
    stot.windows += sst.windows;
    stot.windows_skipped += sst.windows_skipped;
    stot.kmers_generated += sst.kmers_generated;
    stot.windows_at_cap += sst.windows_at_cap;
    stot.exact_seeds_added += sst.exact_seeds_added;
    stot.seeds += sst.seeds;
    stot.postings_visited += sst.postings_visited;
    stot.seeds_over_occ_cap += sst.seeds_over_occ_cap;
    stot.postings_skipped_occ += sst.postings_skipped_occ;
    TraceClock tc("search chunk");
    if (nh) {
      DevMem cm;
      ST_TRY(pool_get(c, static_cast<size_t>(nh) * sizeof(GateCandidate), cm));
      tc.lap("candidate buffer");
      GateStats st{};
      uint64_t nc = 0;
      ST_TRY(gate_pipeline(c, hits.as<GateSeedHit>(), nh, gc, qbits, cm.as<GateCandidate>(), &nc, &st));
      tc.lap("gate");
      const size_t at = all.size();
      all.resize(at + nc);
      if (nc) ST_CUDA(cudaMemcpyAsync(all.data() + at, cm.p, nc * sizeof(st_candidate), cudaMemcpyDeviceToHost,
                                      c->stream));
      ST_CUDA(cudaStreamSynchronize(c->stream));
      pool_put(c, std::move(cm));
      tc.lap("candidates to host");
      tot.targets_hit += st.targets_hit;
      tot.targets_evaluated += st.targets_evaluated;
      tot.diagonals_scored += st.diagonals_scored;
      tot.chains_used += st.chains_used;
      tot.candidates += st.candidates;
      tot.candidates_capped += st.candidates_capped;
      tot.hits_rejected += st.hits_rejected;
    }
    pool_put(c, std::move(hits));
    q0 = q1;
  }
  // chunks are ranked by query id inside themselves; a counting sort by query id (stable) orders the whole
  // list, straight into the caller's buffer
  if (seed_stats) *seed_stats = stot;
  *n_out = all.size();
  if (cap && !all.empty()) {
    std::vector<st_candidate> tmp;
    st_candidate* dst = out;
    if (cap < all.size()) {  // only the first cap are wanted
      tmp.resize(all.size());
      dst = tmp.data();
    }
    std::vector<uint64_t> at(c->profs.size() + 1, 0);
    for (const st_candidate& x : all) ++at[x.query + 1];
    for (size_t i = 1; i < at.size(); ++i) at[i] += at[i - 1];
    for (const st_candidate& x : all) dst[at[x.query]++] = x;
    if (dst != out) memcpy(out, dst, cap * sizeof(st_candidate));
  }
  return gate_result(tot, stats);
}

// ---------------------------------------------------------------------------
// per-profile calibration (st_calib.cuh)
// ---------------------------------------------------------------------------
// The context's database, swapped out while calibration targets take its place
// for one batched scoring call (the planner and the kernels read the context's
// database; kernels already queued keep the pointers they were launched with).
struct DbState {
  DevMem arena, off, len;
  std::vector<uint32_t> h_len;
  std::vector<uint64_t> h_off;
  uint32_t n_seqs = 0, max_len = 0;
  uint64_t n_res = 0;
  bool has = false;
};

// The swapped-in tables may still be filling on the context's stream: the
// event marks that point for work launched on other streams.
static void swap_db(st_ctx* c, DbState& s) {
  if (!c->db_ev && cudaEventCreateWithFlags(&c->db_ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    c->db_ev = nullptr;
    cudaStreamSynchronize(c->stream);  // no event: wait instead
  }
  if (c->db_ev) {
    cudaEventRecord(c->db_ev, c->stream);
    c->db_ev_set = true;
  }
  std::swap(c->db_arena, s.arena);
  std::swap(c->db_off, s.off);
  std::swap(c->db_len, s.len);
  std::swap(c->h_db_len, s.h_len);
  std::swap(c->h_db_off, s.h_off);
  std::swap(c->n_seqs, s.n_seqs);
  std::swap(c->max_len, s.max_len);
  std::swap(c->n_res, s.n_res);
  std::swap(c->has_db, s.has);
}

// fit_gumbel_ml and gumbel_mu_given_lambda (src/evalue.rs:129-182) in binary64
// with the reference's summation order (index order).
static double gumbel_mu_given_lambda(const std::vector<double>& xs, double lambda) {
  double xmin = INFINITY;
  for (double x : xs) xmin = std::fmin(xmin, x);
  double s = 0.0;
  for (double x : xs) s += std::exp(-lambda * (x - xmin));
  return xmin - std::log(s / static_cast<double>(xs.size())) / lambda;
}

static bool fit_gumbel_ml(const std::vector<double>& xs, double* lambda, double* mu) {
  const size_t n = xs.size();
  if (n < 10) return false;
  double sum = 0.0;
  for (double x : xs) sum += x;
  const double mean = sum / static_cast<double>(n);
  double ss = 0.0;
  for (double x : xs) ss += (x - mean) * (x - mean);
  const double var = ss / (static_cast<double>(n) - 1.0);
  if (std::isnan(var) || var <= 0.0) return false;
  double xmin = INFINITY;
  for (double x : xs) xmin = std::fmin(xmin, x);
  auto g = [&](double lam) {
    double s0 = 0.0, s1 = 0.0;
    for (double x : xs) {
      const double w = std::exp(-lam * (x - xmin));
      s0 += w;
      s1 += x * w;
    }
    return 1.0 / lam - mean + s1 / s0;
  };
  const double kPi = 3.141592653589793238462643383279502884;
  const double lam0 = kPi / (std::sqrt(var) * std::sqrt(6.0));
  double lo = lam0 / 10.0, hi = lam0 * 10.0;
  if (g(lo) < 0.0 || g(hi) > 0.0) return false;
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (g(mid) > 0.0)
      lo = mid;
    else
      hi = mid;
    if (hi - lo < 1e-12 * hi) break;
  }
  *lambda = 0.5 * (lo + hi);
  *mu = gumbel_mu_given_lambda(xs, *lambda);
  return true;
}

extern "C" int st_calibrate_profiles(st_ctx* c, const uint32_t* profiles, uint32_t n_profiles, const uint32_t* lengths,
                                     uint32_t n_lengths, uint32_t samples, uint64_t seed, const double* p_back,
                                     int32_t open, int32_t ext, int32_t* scores, st_calibration* out) {
  CTX_GUARD(c);
  if ((n_profiles && (!profiles || !out)) || (n_lengths && !lengths) || !p_back)
    return fail(ST_EINVAL, "st_calibrate_profiles: null argument");
  std::vector<uint32_t> m(n_profiles);
  for (uint32_t i = 0; i < n_profiles; ++i) {
    ST_TRY(check_profile(c, profiles[i]));
    m[i] = c->profs[profiles[i]].m;
    out[i] = st_calibration{0.0, 0.0, 0.0, samples, 0};
  }
  if (n_lengths == 0 || samples == 0 || n_profiles == 0) return ST_OK;  // the reference returns None
  ST_TRY(sync_profiles(c));
  // BackgroundSampler::new (src/evalue.rs:90-100)
  CalibGen gen;
  {
    double total = 0.0;
    for (int i = 0; i < 20; ++i) total += p_back[i];
    double acc = 0.0;
    for (int i = 0; i < 20; ++i) {
      acc += p_back[i] / total;
      gen.cum[i] = acc;
    }
    gen.cum[19] = 1.0;
  }
  // per sample: stream seed, length draw, layout
  DbState cal;
  cal.h_len.resize(samples);
  cal.h_off.resize(samples);
  std::vector<uint64_t> state(samples), off(static_cast<size_t>(samples) + 1);
  uint64_t total = 0;
  for (uint32_t i = 0; i < samples; ++i) {
    uint64_t s = seed ^ (0xBEEFull * 0xA24BAED4963EE407ull) ^ (static_cast<uint64_t>(i) * 0x9FB21C651E98DF25ull);
    s += kSplitMixGamma;
    s = splitmix_mix(s);  // stream_seed: the first output of the derived generator
    s += kSplitMixGamma;
    const uint32_t n = std::max<uint32_t>(lengths[splitmix_mix(s) % n_lengths], 1u);
    state[i] = s;
    cal.h_len[i] = n;
    cal.h_off[i] = total;
    off[i] = total;
    cal.max_len = std::max(cal.max_len, n);
    cal.n_res += n;
    total += up16(n);
  }
  off[samples] = total;
  cal.n_seqs = samples;
  cal.has = true;
  const size_t arena_bytes = total + 32;
  ST_TRY(dev_alloc(&c->mt, cal.arena, arena_bytes));
  ST_TRY(dev_alloc(&c->mt, cal.off, off.size() * 8));
  ST_TRY(dev_alloc(&c->mt, cal.len, static_cast<size_t>(samples) * 4));
  DevMem st_dev;
  ST_TRY(pool_get(c, static_cast<size_t>(samples) * 8, st_dev));
  ST_CUDA(cudaMemsetAsync(cal.arena.p, kSentinel, arena_bytes, c->stream));
  ST_CUDA(cudaMemcpyAsync(cal.off.p, off.data(), off.size() * 8, cudaMemcpyHostToDevice, c->stream));
  ST_CUDA(cudaMemcpyAsync(cal.len.p, cal.h_len.data(), static_cast<size_t>(samples) * 4, cudaMemcpyHostToDevice,
                          c->stream));
  ST_CUDA(cudaMemcpyAsync(st_dev.p, state.data(), static_cast<size_t>(samples) * 8, cudaMemcpyHostToDevice,
                          c->stream));
  gen.state = st_dev.as<uint64_t>();
  gen.offset = cal.off.as<uint64_t>();
  gen.length = cal.len.as<uint32_t>();
  gen.arena = cal.arena.as<uint8_t>();
  calib_targets_kernel<<<samples, 256, 0, c->stream>>>(gen);
  ++c->launches;
  ST_CUDA(cudaGetLastError());
  // every (profile, sample) pair in one batched call against the calibration targets
  std::vector<st_pair> pairs;
  std::vector<uint32_t> row;  // profile index of each block of `samples` pairs
  pairs.reserve(static_cast<size_t>(n_profiles) * samples);
  for (uint32_t p = 0; p < n_profiles; ++p) {
    if (m[p] == 0) continue;  // the reference returns None for an empty table
    row.push_back(p);
    for (uint32_t i = 0; i < samples; ++i) pairs.push_back(st_pair{profiles[p], i, 0, -1});
  }
  std::vector<int32_t> sc(pairs.size());
  uint64_t lsum = 0;
  for (uint32_t i = 0; i < n_lengths; ++i) lsum += lengths[i];
  const double mean_len = static_cast<double>(lsum) / static_cast<double>(n_lengths);
  // ML Gumbel fit per profile, K over the search space m * (N_t * mean length) (src/evalue.rs:739-747)
  auto fit_rows = [&](size_t r0, size_t r1) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t r = static_cast<int64_t>(r0); r < static_cast<int64_t>(r1); ++r) {
      std::vector<double> xs(samples);
      for (uint32_t i = 0; i < samples; ++i) xs[i] = static_cast<double>(sc[static_cast<size_t>(r) * samples + i]);
      double lambda = 0.0, mu = 0.0;
      st_calibration& o = out[row[r]];
      if (fit_gumbel_ml(xs, &lambda, &mu)) {
        o.lambda = lambda;
        o.mu = mu;
        o.k = std::exp(lambda * (mu + 0.5)) / (static_cast<double>(m[row[r]]) * mean_len);
        o.ok = 1;
      }
    }
  };
  // profiles in groups: group g + 1 is scored on the device while the host fits group g
  const size_t n_rows = row.size();
  const size_t per = std::max<size_t>(64, (n_rows + 3) / 4);
  std::vector<size_t> gs;
  for (size_t r = 0; r < n_rows; r += per) gs.push_back(r);
  gs.push_back(n_rows);
  const size_t ng = gs.size() - 1;
  std::vector<st_batch*> handles(ng, nullptr);
  auto launch = [&](size_t g) {
    const size_t a = gs[g] * samples, b = gs[g + 1] * samples;
    return st_sw_score_pairs_async(c, pairs.data() + a, b - a, open, ext, sc.data() + a, nullptr, &handles[g]);
  };
  swap_db(c, cal);
  int rc = ng ? launch(0) : ST_OK;
  for (size_t g = 0; g < ng && rc == ST_OK; ++g) {
    if (g + 1 < ng) {
      rc = launch(g + 1);
      if (rc != ST_OK) break;
    }
    rc = st_batch_wait(handles[g]);
    handles[g] = nullptr;
    if (rc == ST_OK) fit_rows(gs[g], gs[g + 1]);
  }
  for (st_batch* h : handles)  // after an error: the batches still in flight
    if (h) st_batch_wait(h);
  swap_db(c, cal);
  ST_CUDA(cudaStreamSynchronize(c->stream));
  pool_put(c, std::move(st_dev));
  if (rc != ST_OK) return rc;
  if (scores) {
    memset(scores, 0, static_cast<size_t>(n_profiles) * samples * 4);
    for (size_t r = 0; r < row.size(); ++r)
      memcpy(scores + static_cast<size_t>(row[r]) * samples, sc.data() + r * samples, static_cast<size_t>(samples) * 4);
  }
  return ST_OK;
}

// ---------------------------------------------------------------------------
// DPX throughput probe (denominator of the SW roofline)
// ---------------------------------------------------------------------------
constexpr int kProbeChains = 8;
constexpr int kProbeIters = 4096;

__global__ void dpx_probe_kernel(uint32_t* sink, uint32_t seed) {
  uint32_t a[kProbeChains];
#pragma unroll
  for (int k = 0; k < kProbeChains; ++k) a[k] = seed * (threadIdx.x + k + 1);
  const uint32_t b = seed ^ 0x00050003u, cc = seed ^ 0x00020001u;
  for (int i = 0; i < kProbeIters; ++i) {
#pragma unroll
    for (int k = 0; k < kProbeChains; ++k) a[k] = __viaddmax_s16x2(a[k], b, cc);
  }
  uint32_t r = 0;
#pragma unroll
  for (int k = 0; k < kProbeChains; ++k) r ^= a[k];
  if (r == 0x9E3779B9u) sink[0] = r;  // keeps the chains live
}

extern "C" int st_probe_dpx(st_ctx* c, double* ops_per_s) {
  CTX_GUARD(c);
  if (!ops_per_s) return fail(ST_EINVAL, "null output");
  DevMem sink;
  ST_TRY(dev_alloc(&c->mt, sink, 16));
  const int blocks = c->sms * 8, threads = 256;
  cudaEvent_t e0, e1;
  ST_CUDA(cudaEventCreate(&e0));
  ST_CUDA(cudaEventCreate(&e1));
  dpx_probe_kernel<<<blocks, threads, 0, c->stream>>>(sink.as<uint32_t>(), 7);
  ST_CUDA(cudaEventRecord(e0, c->stream));
  const int reps = 5;
  for (int r = 0; r < reps; ++r) dpx_probe_kernel<<<blocks, threads, 0, c->stream>>>(sink.as<uint32_t>(), 11 + r);
  ST_CUDA(cudaEventRecord(e1, c->stream));
  ST_CUDA(cudaEventSynchronize(e1));
  c->launches += reps + 1;
  float ms = 0;
  ST_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const double ops = static_cast<double>(reps) * blocks * threads * kProbeIters * kProbeChains;
  *ops_per_s = ops / (ms * 1e-3);
  return ST_OK;
}

// ---------------------------------------------------------------------------
// tile classes and the autotuner
// ---------------------------------------------------------------------------
extern "C" int st_tune_num_classes(void) { return kNumClasses; }

extern "C" int st_tune_class_shape(int cls, int* lanes, int* rows, int* cols) {
  if (cls < 0 || cls >= kNumClasses || !lanes || !rows) return fail(ST_EINVAL, "bad tile class %d", cls);
  *lanes = kClasses[cls].G;
  *rows = kClasses[cls].R;
  if (cols) *cols = kClasses[cls].C;
  return ST_OK;
}

extern "C" int st_tune_get(st_ctx* c, int32_t* table) {
  CTX_GUARD(c);
  if (!table) return fail(ST_EINVAL, "null table");
  for (int i = 0; i < kTuneMBins; ++i)
    for (int j = 0; j < kTuneNBins; ++j) table[i * kTuneNBins + j] = c->tuning.table[i][j];
  return ST_OK;
}

extern "C" int st_tune_set(st_ctx* c, const int32_t* table) {
  CTX_GUARD(c);
  if (!table) return fail(ST_EINVAL, "null table");
  for (int i = 0; i < kTuneMBins * kTuneNBins; ++i)
    if (table[i] < -1 || table[i] >= kNumClasses) return fail(ST_EINVAL, "bad class %d in table", table[i]);
  for (int i = 0; i < kTuneMBins; ++i)
    for (int j = 0; j < kTuneNBins; ++j) c->tuning.table[i][j] = table[i * kTuneNBins + j];
  return ST_OK;
}

// Calibrates the rate of every 16-bit tile class on a sample of the batch:
// whole queries, spread over the batch, up to max_pairs pairs. The sample is
// planned with every query forced into one class at a time, timed (one
// warm-up run, then three), and the class's rate set to the streamed cells
// per second. The forcing table is restored afterwards.
extern "C" int st_autotune(st_ctx* c, const st_pair* pairs, uint64_t n, int32_t open, int32_t ext,
                           uint32_t max_pairs, uint32_t* classes_calibrated) {
  CTX_GUARD(c);
  if (n && !pairs) return fail(ST_EINVAL, "st_autotune: null pairs");
  if (!c->has_db) return fail(ST_ESTATE, "no target database uploaded (st_db_upload)");
  ST_TRY(sync_profiles(c));
  if (classes_calibrated) *classes_calibrated = 0;
  if (!gaps16_ok(open, ext)) return ST_OK;  // nothing runs on the 16-bit kernel
  // queries that every class can stage (the models' shared-memory limit)
  uint32_t max_m = UINT32_MAX;
  for (int k = 0; k < kNumClasses; ++k) {
    const uint32_t rows = static_cast<uint32_t>(kClasses[k].G * kClasses[k].R);
    max_m = std::min(max_m, static_cast<uint32_t>(216 * 1024) / kProfRows / rows * rows);
  }
  std::vector<std::vector<uint32_t>> byq(c->profs.size());
  for (uint64_t i = 0; i < n; ++i) {
    const st_pair& p = pairs[i];
    if (p.profile >= c->profs.size() || !c->profs[p.profile].live || p.target >= c->n_seqs)
      return fail(ST_EINVAL, "st_autotune: bad pair %llu", static_cast<unsigned long long>(i));
    const ProfileMeta& pm = c->profs[p.profile];
    if (p.band_radius >= 0 || !pm.fits8 || pm.m == 0 || pm.m > max_m || c->h_db_len[p.target] == 0) continue;
    byq[p.profile].push_back(static_cast<uint32_t>(i));
  }
  std::vector<uint32_t> qs;
  for (uint32_t q = 0; q < byq.size(); ++q)
    if (!byq[q].empty()) qs.push_back(q);
  if (qs.empty()) return ST_OK;
  // whole queries in a fixed scattered order (a multiplicative hash of the id) until the sample is full
  std::sort(qs.begin(), qs.end(), [](uint32_t a, uint32_t b) { return a * 2654435761u < b * 2654435761u; });
  std::vector<st_pair> sample;
  for (size_t k = 0; k < qs.size() && sample.size() < max_pairs; ++k)
    for (uint32_t i : byq[qs[k]]) sample.push_back(pairs[i]);
  DevMem out;
  ST_TRY(dev_alloc(&c->mt, out, sample.size() * 8));
  cudaEvent_t e0, e1;
  ST_CUDA(cudaEventCreate(&e0));
  ST_CUDA(cudaEventCreate(&e1));
  struct Events {
    cudaEvent_t a, b;
    ~Events() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } evs{e0, e1};
  Tuning saved = c->tuning;
  struct Restore {
    st_ctx* c;
    Tuning* t;
    bool armed = true;
    ~Restore() {
      if (armed) c->tuning = *t;
    }
  } restore{c, &saved};
  float rates[kMaxTileClasses] = {};
  uint32_t done = 0;
  for (int k = 0; k < kNumClasses; ++k) {
    for (int i = 0; i < kTuneMBins; ++i)
      for (int j = 0; j < kTuneNBins; ++j) c->tuning.table[i][j] = k;
    st_plan* p = nullptr;
    ST_TRY(plan_build(c, sample.data(), sample.size(), open, ext, out.as<int32_t>(), nullptr, &p, true, c->own, 0));
    std::unique_ptr<st_plan, void (*)(st_plan*)> guard(p, plan_free);
    cudaStream_t prev = c->stream;
    c->stream = c->own;
    int rc = plan_run(p);  // warm-up
    if (rc == ST_OK && cudaEventRecord(e0, c->own) != cudaSuccess) rc = fail(ST_ECUDA, "event record failed");
    for (int r = 0; r < 3 && rc == ST_OK; ++r) rc = plan_run(p);
    if (rc == ST_OK && cudaEventRecord(e1, c->own) != cudaSuccess) rc = fail(ST_ECUDA, "event record failed");
    c->stream = prev;
    ST_TRY(rc);
    ST_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    ST_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms > 0 && p->streamed > 0) {
      rates[k] = static_cast<float>(static_cast<double>(p->streamed) * 3 / (ms * 1e-3) / 1e12);
      ++done;
    }
  }
  for (int k = 0; k < kNumClasses; ++k) saved.rate[k] = rates[k];
  if (classes_calibrated) *classes_calibrated = done;
  return ST_OK;
}

extern "C" int st_tune_get_rates(st_ctx* c, float* rates, uint32_t cap) {
  CTX_GUARD(c);
  if (cap && !rates) return fail(ST_EINVAL, "st_tune_get_rates: null output");
  for (uint32_t k = 0; k < cap && k < static_cast<uint32_t>(kNumClasses); ++k) rates[k] = c->tuning.rate[k];
  return ST_OK;
}

extern "C" int st_tune_set_rates(st_ctx* c, const float* rates, uint32_t n) {
  CTX_GUARD(c);
  if (n && !rates) return fail(ST_EINVAL, "st_tune_set_rates: null input");
  if (n > static_cast<uint32_t>(kNumClasses)) return fail(ST_EINVAL, "st_tune_set_rates: %u rates for %d classes", n, kNumClasses);
  for (uint32_t k = 0; k < n; ++k) {
    if (!(rates[k] >= 0.0f) || rates[k] > 1e6f) return fail(ST_EINVAL, "st_tune_set_rates: bad rate %g", rates[k]);
    c->tuning.rate[k] = rates[k];
  }
  return ST_OK;
}
