// Prefilter evidence, chaining and gate on the device: the reference's
// segment-evidence stage (xdrop = 0) of prefilter_query, src/prefilter.rs:
//   evaluate_block_kadane  :1412-1493  group hits by target, keep the
//                                      max_diagonals diagonals with the most hits
//                                      (top_diagonals :1194-1225), one job per
//                                      diagonal with its window
//   score_and_gate         :1498-1660  best ungapped segment per job, best single
//                                      segment or chain of two co-linear
//                                      segments, gate, region
//   ranking                :1074-1083  score descending, target ascending,
//                                      max_candidates per query
// for many queries at once.  Pipeline (one stream, no host round trip):
//   keys     one thread per hit: key = (query, target, diagonal + max_m), value =
//            query position; hits outside the query or the target get the key
//            of a query id past the last profile (they sort last and are skipped)
//   sort     radix sort of the keys (CUB)
//   groups   start of each (query, target) run of the sorted keys (CUB select)
//   count    one thread per group: min_hits / diag_hits tests and the number of
//            jobs, min(distinct diagonals, max_diagonals, 16)
//   scan     job offsets (CUB exclusive sum)
//   emit     one thread per group: the top diagonals by hit count (stable on the
//            ascending diagonal order) and their windows, written as jobs
//   score    one job per lane with refill, jobs of one query share its profile
//            staged in shared memory: kadane_score over the window
//   screen   groups that may pass (several diagonals, or one at the gate) to a
//            work list
//   chain    one thread per listed group: best segment, best chain, gate,
//            region, candidate slot + flag; kadane_segment positions only for
//            the jobs a chain test or a region reads (the reference's pos_of)
//   compact  candidates in (query, target) order (CUB select)
//   rank     stable radix sort by (query, 2^31 - 1 - score) keeps target order
//            inside equal scores; per-query cut to max_candidates; gather
#pragma once
#include "st_common.cuh"

namespace st {

constexpr int kGateMaxDiags = 16;  // jobs per target (src/prefilter.rs:1459, top.iter().take(16))
constexpr int kGateChunk = 1024;   // jobs per CTA chunk of the segment kernel

struct GateCandidate {  // the layout of st_candidate
  uint32_t query;
  uint32_t target;
  uint32_t hits;
  int32_t diag_score;
  int64_t best_diag;
  uint32_t t_lo;
  uint32_t t_hi;
};
static_assert(sizeof(GateCandidate) == 32, "candidate layout");

struct GateJob {
  uint32_t query;
  uint32_t target;
  int32_t diag;
  uint32_t lo;
  uint32_t hi;
};

struct GateSeedHit {  // the layout of st_seed_hit
  uint32_t query;
  uint32_t target;
  int32_t diag;
  uint32_t qpos;
};

// Counters, the layout of st_prefilter_stats.
struct GateStats {
  unsigned long long targets_hit;
  unsigned long long targets_evaluated;
  unsigned long long diagonals_scored;
  unsigned long long chains_used;
  unsigned long long candidates;
  unsigned long long candidates_capped;
  unsigned long long hits_rejected;
};

struct GateConf {
  uint32_t min_hits;
  uint32_t diag_hits;
  uint32_t kmax;  // min(max_diagonals, 16)
  uint32_t window;
  uint32_t span;
  int32_t min_score;
  int32_t open;
  int32_t ext;
  uint32_t max_cand;  // 0 = all
  uint32_t regions;
  // key layout: query << (tbits + dbits) | target << dbits | (diag + doff)
  uint32_t tbits;
  uint32_t dbits;
  uint32_t doff;
  uint32_t n_prof;  // query ids are < n_prof; n_prof marks rejected hits
  uint32_t stride;  // staged profile row stride: >= every hit query's length rounded to 16, + 32
};

__device__ __forceinline__ uint32_t gate_key_query(uint64_t k, const GateConf& g) {
  return static_cast<uint32_t>(k >> (g.tbits + g.dbits));
}
__device__ __forceinline__ uint32_t gate_key_target(uint64_t k, const GateConf& g) {
  return static_cast<uint32_t>((k >> g.dbits) & ((1ull << g.tbits) - 1));
}
__device__ __forceinline__ int32_t gate_key_diag(uint64_t k, const GateConf& g) {
  return static_cast<int32_t>(static_cast<int64_t>(k & ((1ull << g.dbits) - 1)) - g.doff);
}

// Adds each thread's count to a counter; called by every thread of the block
// once, after its loop (all 32 lanes of each warp present).
__device__ __forceinline__ void gate_flush(unsigned long long* ctr, unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(ctr, v);
}

__global__ void __launch_bounds__(256) gate_keys_kernel(const GateSeedHit* hits, uint64_t n, DeviceDb db,
                                                        const uint32_t* qlen, GateConf g, uint64_t* keys,
                                                        uint32_t* vals, GateStats* st) {
  const uint64_t bad = static_cast<uint64_t>(g.n_prof) << (g.tbits + g.dbits);
  unsigned long long rejected = 0;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const GateSeedHit h = hits[i];
    bool ok = h.query < g.n_prof && h.target < db.n_seqs;
    if (ok) {
      const int64_t tpos = static_cast<int64_t>(h.qpos) + h.diag;
      ok = h.qpos < qlen[h.query] && tpos >= 0 && tpos < static_cast<int64_t>(db.length[h.target]);
    }
    uint64_t k = bad;
    if (ok)
      k = (static_cast<uint64_t>(h.query) << (g.tbits + g.dbits)) | (static_cast<uint64_t>(h.target) << g.dbits) |
          static_cast<uint64_t>(static_cast<int64_t>(h.diag) + g.doff);
    keys[i] = k;
    vals[i] = h.qpos;
    rejected += ok ? 0 : 1;
  }
  gate_flush(&st->hits_rejected, rejected);
}

// Flag of the first hit of each (query, target) run in the sorted keys.
struct GateHeadFlag {
  const uint64_t* keys;
  uint32_t shift;  // dbits
  __host__ __device__ bool operator()(uint32_t i) const {
    return i == 0 || (keys[i] >> shift) != (keys[i - 1] >> shift);
  }
};

struct GateGroups {
  const uint64_t* keys;  // sorted
  const uint32_t* vals;  // query positions, in key order
  const uint32_t* start; // first hit of each group
  const uint32_t* n_groups;
  uint32_t n_hits;
};

__device__ __forceinline__ void gate_group_range(const GateGroups& G, uint32_t gi, uint32_t ng, uint32_t& s,
                                                 uint32_t& e) {
  s = G.start[gi];
  e = gi + 1 < ng ? G.start[gi + 1] : G.n_hits;
}

// ns[g] = jobs of group g (0 when the target is dropped); entries from the last
// group to n_hits are zeroed so the exclusive sum over n_hits + 1 entries ends
// at the total job count.
__global__ void __launch_bounds__(256) gate_count_kernel(GateGroups G, GateConf g, uint32_t* ns, GateStats* st) {
  const uint32_t ng = *G.n_groups;
  unsigned long long n_hit = 0, n_eval = 0;
  for (uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x; gi <= G.n_hits; gi += gridDim.x * blockDim.x) {
    uint32_t jobs = 0, evaluated = 0, hit = 0;
    if (gi < ng) {
      uint32_t s, e;
      gate_group_range(G, gi, ng, s, e);
      const uint64_t k0 = G.keys[s];
      if (gate_key_query(k0, g) < g.n_prof) {
        hit = 1;
        if (e - s >= g.min_hits) {
          uint32_t runs = 0, best = 0, cnt = 0;
          uint64_t prev = ~0ull;
          for (uint32_t i = s; i < e; ++i) {
            const uint64_t k = G.keys[i];
            if (k != prev) {
              ++runs;
              cnt = 0;
              prev = k;
            }
            ++cnt;
            best = max(best, cnt);
          }
          if (best >= g.diag_hits) {
            jobs = min(runs, g.kmax);
            evaluated = 1;
          }
        }
      }
    }
    ns[gi] = jobs;
    n_hit += hit;
    n_eval += evaluated;
  }
  gate_flush(&st->targets_hit, n_hit);
  gate_flush(&st->targets_evaluated, n_eval);
}

struct GateRun {
  int32_t diag;
  uint32_t count;
  uint32_t qmin;
  uint32_t qmax;
};

// Jobs of each kept group: its KMAX best diagonals by hit count (a run goes
// before the first kept run with a smaller count, so equal counts keep the
// ascending diagonal order), with windows (src/prefilter.rs:1459-1474).
template <int KMAX>
__global__ void __launch_bounds__(128) gate_emit_kernel(GateGroups G, GateConf g, DeviceDb db, const uint32_t* qlen,
                                                        const uint32_t* ns, const uint32_t* joff, GateJob* jobs) {
  const uint32_t ng = *G.n_groups;
  for (uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x; gi < ng; gi += gridDim.x * blockDim.x) {
    if (ns[gi] == 0) continue;
    uint32_t s, e;
    gate_group_range(G, gi, ng, s, e);
    GateRun top[KMAX];
    uint32_t nt = 0;
    uint32_t i = s;
    while (i < e) {
      const uint64_t k = G.keys[i];
      GateRun r{gate_key_diag(k, g), 0, G.vals[i], G.vals[i]};
      uint32_t j = i;
      for (; j < e && G.keys[j] == k; ++j) {
        r.qmin = min(r.qmin, G.vals[j]);
        r.qmax = max(r.qmax, G.vals[j]);
      }
      r.count = j - i;
      i = j;
      // pos = kept runs with count >= r.count
      uint32_t pos = 0;
#pragma unroll
      for (int t = 0; t < KMAX; ++t) pos += (static_cast<uint32_t>(t) < nt && top[t].count >= r.count) ? 1u : 0u;
      if (pos < g.kmax) {
#pragma unroll
        for (int t = KMAX - 1; t > 0; --t)
          if (static_cast<uint32_t>(t) > pos) top[t] = top[t - 1];
#pragma unroll
        for (int t = 0; t < KMAX; ++t)
          if (static_cast<uint32_t>(t) == pos) top[t] = r;
        nt = min(nt + 1, g.kmax);
      }
    }
    const uint64_t k0 = G.keys[s];
    const uint32_t q = gate_key_query(k0, g), t = gate_key_target(k0, g);
    const int64_t m = qlen[q], n = db.length[t];
    GateJob* out = jobs + joff[gi];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
      if (static_cast<uint32_t>(k) >= nt) break;
      const int32_t d = top[k].diag;
      // diag_range (src/ungapped.rs:38-46), then the window around the hits
      int64_t lo = i64max(-static_cast<int64_t>(d), 0), hi = i64min(m, n - d);
      if (hi <= lo) lo = hi = 0;
      if (g.window > 0) {
        const int64_t a = top[k].qmin > g.window ? static_cast<int64_t>(top[k].qmin - g.window) : 0;
        const int64_t b = static_cast<int64_t>(top[k].qmax) + g.span + g.window;
        lo = i64max(lo, a);
        hi = i64min(hi, b);
      }
      hi = i64max(hi, lo);
      out[k] = GateJob{q, t, d, static_cast<uint32_t>(lo), static_cast<uint32_t>(hi)};
    }
  }
}

struct GateSegParams {
  DeviceDb db;
  DeviceProfiles prof;
  const GateJob* jobs;
  const uint32_t* n_groups;
  const uint32_t* joff;  // total jobs at joff[n_groups]
  int32_t* score;
  uint32_t max_m_pad;
};

// Byte mask of a 16-byte vector: 0xFF for the bytes i with lo <= i < hi.
__device__ __forceinline__ void gate_window_mask(int32_t lo, int32_t hi, uint32_t m[4]) {
  const uint32_t bits = ((1u << hi) - 1u) & ~((1u << lo) - 1u);  // 0 <= lo < hi <= 16
#pragma unroll
  for (int j = 0; j < 4; ++j) m[j] = (((bits >> (4 * j)) & 0xFu) * 0x00204081u & 0x01010101u) * 0xFFu;
}

// kadane_score (src/ungapped.rs:53-62) of each job over its window.  A CTA
// takes a chunk of jobs; per run of one query inside it the query's int8
// profile is staged in shared memory and every thread keeps one job in flight,
// one 16-byte target vector per step, taking the run's next job (shared
// counter) as soon as its own is done, so lanes stay busy whatever the window
// lengths.  The first and last vectors of a window have their bytes outside
// the window replaced by the sentinel code, whose profile row is zero: zero
// cells at the ends of a window change no Kadane maximum, so the cell loop has
// no window test.  Profiles outside int8 read int32 rows from global memory
// with an explicit test.
__global__ void __launch_bounds__(256) gate_score_kernel(const GateSegParams prm) {
  extern __shared__ __align__(16) int8_t smem[];
  __shared__ uint32_t s_run_end, s_next;
  const uint32_t n = prm.joff[*prm.n_groups];
  const uint32_t stride = prm.max_m_pad;
  int8_t* base = smem + 16;
  const uint32_t c0 = blockIdx.x * kGateChunk;
  if (c0 >= n) return;
  const uint32_t c1 = min(n, c0 + kGateChunk);
  uint32_t a = c0;
  while (a < c1) {
    const uint32_t q = prm.jobs[a].query;
    if (threadIdx.x < 32) {
      uint32_t e = a;
      for (;;) {
        const uint32_t k = e + threadIdx.x;
        const bool same = (k < c1) && (prm.jobs[k].query == q);
        const uint32_t ball = __ballot_sync(0xFFFFFFFFu, same);
        if (ball != 0xFFFFFFFFu) {
          e += __ffs(~ball) - 1;
          break;
        }
        e += 32;
      }
      if (threadIdx.x == 0) {
        s_run_end = e;
        s_next = a + blockDim.x;
      }
    }
    const uint32_t pstride = prm.prof.stride8[q];
    const int8_t* src = prm.prof.p8[q];
    for (uint32_t idx = threadIdx.x; idx < kProfRows * (stride / 16); idx += blockDim.x) {
      const uint32_t r = idx / (stride / 16);
      const uint32_t i = (idx - r * (stride / 16)) * 16;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (i < pstride) v = *reinterpret_cast<const uint4*>(src + static_cast<size_t>(r) * pstride + i);
      *reinterpret_cast<uint4*>(base + static_cast<size_t>(r) * stride + i) = v;
    }
    if (threadIdx.x < 16) smem[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t b = s_run_end;
    const bool narrow = prm.prof.fits8[q] != 0;
    const int32_t* p32 = prm.prof.p32[q];
    const int32_t s32 = static_cast<int32_t>(prm.prof.stride32[q]);
    const int32_t last_row = static_cast<int32_t>(prm.prof.qlen[q]) - 1;
    // per lane: job k, target base, diagonal, window [p0, p1) in target positions, next vector pa
    uint32_t k = a + threadIdx.x;
    const uint8_t* tp = nullptr;
    int32_t d = 0, p0 = 0, p1 = 0, pa = 0, cur = 0, best = 0;
    bool live = false;
    auto take = [&](uint32_t j) {
      k = j;
      live = j < b;
      if (live) {
        const GateJob jb = prm.jobs[j];
        tp = prm.db.arena + prm.db.offset[jb.target];
        d = jb.diag;
        p0 = static_cast<int32_t>(jb.lo) + d;
        p1 = static_cast<int32_t>(jb.hi) + d;
        pa = jb.hi > jb.lo ? (p0 & ~15) : p1;  // an empty window is done at once (p0 may be negative)
        cur = 0;
        best = 0;
      }
    };
    take(k);
    while (__any_sync(0xFFFFFFFFu, live)) {
      if (live) {
        if (pa < p1) {
          const uint4 v = *reinterpret_cast<const uint4*>(tp + pa);
          uint32_t w[4] = {v.x, v.y, v.z, v.w};
          const int32_t qa = pa - d;
          if (narrow) {
            if (pa < p0 || pa + 16 > p1) {  // a window end inside this vector
              uint32_t m[4];
              gate_window_mask(max(p0 - pa, 0), min(p1 - pa, 16), m);
#pragma unroll
              for (int j = 0; j < 4; ++j) w[j] = (w[j] & m[j]) | (0x15151515u & ~m[j]);
            }
            const int8_t* rowbase = base + qa;
#pragma unroll
            for (int bb = 0; bb < 16; ++bb) {
              const uint32_t r = (w[bb >> 2] >> ((bb & 3) * 8)) & 0xFFu;
              cur = wadd(max(cur, 0), static_cast<int32_t>(rowbase[static_cast<int32_t>(r * stride) + bb]));
              best = max(best, cur);
            }
          } else {
#pragma unroll
            for (int bb = 0; bb < 16; ++bb) {
              const uint32_t r = (w[bb >> 2] >> ((bb & 3) * 8)) & 0xFFu;
              const int32_t p = pa + bb;
              const int32_t row = min(max(qa + bb, 0), last_row);
              const int32_t sc = (p >= p0 && p < p1) ? __ldg(p32 + static_cast<int32_t>(r) * s32 + row) : 0;
              cur = wadd(max(cur, 0), sc);
              best = max(best, cur);
            }
          }
          pa += 16;
        }
        if (pa >= p1) {  // done (or an empty window)
          prm.score[k] = best;
          take(atomicAdd(&s_next, 1u));
        }
      }
    }
    __syncthreads();
    a = b;
  }
}

// kadane_segment (src/ungapped.rs:69-88) of one job from the profile in global
// memory: best score, start of the run that first reaches it and its end
// (0, 0 when the best is 0).  Used only for the jobs whose positions decide a
// chain or a region.  Target residues come as 16-byte vectors and the 16
// profile loads of a vector are independent of each other; cells outside the
// window score 0, which moves neither the best nor where it is first reached.
__device__ int32_t gate_kadane_segment(const DeviceProfiles& prof, const DeviceDb& db, const GateJob& jb, int32_t& qs,
                                       int32_t& qe) {
  int32_t best = 0, cur = 0, bs = 0, be = 0, cs = 0;
  if (jb.hi > jb.lo) {
    const uint8_t* t = db.arena + db.offset[jb.target];
    const bool narrow = prof.fits8[jb.query] != 0;
    const int8_t* p8 = prof.p8[jb.query];
    const int32_t* p32 = prof.p32[jb.query];
    const int32_t s8 = static_cast<int32_t>(prof.stride8[jb.query]), s32 = static_cast<int32_t>(prof.stride32[jb.query]);
    const int32_t d = jb.diag, lo = static_cast<int32_t>(jb.lo), hi = static_cast<int32_t>(jb.hi);
    const int32_t p0 = lo + d, p1 = hi + d;
    for (int32_t pa = p0 & ~15; pa < p1; pa += 16) {
      const uint4 v = *reinterpret_cast<const uint4*>(t + pa);
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int bb = 0; bb < 16; ++bb) {
        const uint32_t r = (w[bb >> 2] >> ((bb & 3) * 8)) & 0xFFu;
        const int32_t q = pa + bb - d;
        const bool in = q >= lo && q < hi;
        const int32_t qc = min(max(q, lo), hi - 1);
        const int32_t sv = narrow ? static_cast<int32_t>(p8[static_cast<int32_t>(r) * s8 + qc])
                                  : p32[static_cast<int32_t>(r) * s32 + qc];
        const int32_t s = in ? sv : 0;
        if (cur <= 0) {
          cur = s;
          cs = q;
        } else {
          cur = wadd(cur, s);
        }
        if (cur > best) {
          best = cur;
          bs = cs;
          be = q;
        }
      }
    }
  }
  qs = bs;
  qe = be;
  return best;
}

__device__ __forceinline__ int32_t gate_gap_cost(int32_t open, int32_t ext, uint32_t len) {
  return len == 0 ? 0 : wadd(open, static_cast<int32_t>((len - 1u) * static_cast<uint32_t>(ext)));
}

// Groups that may pass the gate: every group with more than one diagonal or
// with its one diagonal at or above the gate goes to a work list (the order of
// the list does not matter: each group writes its own slot).  Groups left out
// keep the zero flag written before.
__global__ void __launch_bounds__(256) gate_screen_kernel(GateGroups G, GateConf g, const uint32_t* joff,
                                                          const int32_t* score, uint32_t* work, uint32_t* n_work) {
  const uint32_t ng = *G.n_groups;
  for (uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x; gi < ng; gi += gridDim.x * blockDim.x) {
    const uint32_t j0 = joff[gi], nsg = joff[gi + 1] - j0;
    if (nsg > 0 && !(nsg == 1 && score[j0] < g.min_score)) work[atomicAdd(n_work, 1u)] = gi;
  }
}

// Best single segment (first maximum in job order) or best chain x -> y of two
// co-linear segments (first maximum in (x, y) order), the gate and the region
// (src/prefilter.rs:1577-1657, region :1269-1278), one thread per listed group.
__global__ void __launch_bounds__(128) gate_chain_kernel(GateGroups G, GateConf g, DeviceDb db, DeviceProfiles prof,
                                                         const uint32_t* joff, const GateJob* jobs,
                                                         const int32_t* score, const uint32_t* work,
                                                         const uint32_t* n_work, GateCandidate* cand, uint8_t* flag,
                                                         GateStats* st) {
  const uint32_t ng = *G.n_groups;
  const uint32_t nw = *n_work;
  unsigned long long n_chained = 0;
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
    const uint32_t gi = work[w];
    const uint32_t j0 = joff[gi], nsg = joff[gi + 1] - j0;
    int32_t best = 0;
    uint32_t bi = 0;
    for (uint32_t k = 0; k < nsg; ++k) {
      const int32_t sk = score[j0 + k];
      if (sk > best) {
        best = sk;
        bi = k;
      }
    }
    // segment positions, computed where a chain or a region needs them (as the reference's pos_of)
    int32_t pqs[kGateMaxDiags], pqe[kGateMaxDiags];
    uint32_t have = 0;
    auto pos_of = [&](uint32_t x) {
      if (!(have & (1u << x))) {
        gate_kadane_segment(prof, db, jobs[j0 + x], pqs[x], pqe[x]);
        have |= 1u << x;
      }
    };
    int32_t chain = INT32_MIN;
    uint32_t cx = 0, cy = 0;
    if (nsg > 1) {
      for (uint32_t x = 0; x < nsg; ++x) {
        const int32_t sx = score[j0 + x];
        if (sx <= 0) continue;
        const int32_t dx = jobs[j0 + x].diag;
        for (uint32_t y = 0; y < nsg; ++y) {
          if (x == y) continue;
          const int32_t sy = score[j0 + y], dy = jobs[j0 + y].diag;
          if (sy <= 0 || dx == dy) continue;
          const uint32_t len = static_cast<uint32_t>(dy > dx ? dy - dx : dx - dy);
          const int32_t c = wsub(wadd(sx, sy), gate_gap_cost(g.open, g.ext, len));
          if (c <= best || c <= chain) continue;
          pos_of(x);
          pos_of(y);
          const int32_t qex = pqe[x], qsy = pqs[y];
          if (qex < qsy && static_cast<int64_t>(qex) + dx < static_cast<int64_t>(qsy) + dy) {
            chain = c;
            cx = x;
            cy = y;
          }
        }
      }
    }
    int32_t total;
    uint32_t u0, u1;
    if (chain > best) {
      ++n_chained;
      total = chain;
      u0 = cx;
      u1 = cy;
    } else {
      total = best;
      u0 = u1 = bi;
    }
    if (total < g.min_score) continue;
    uint32_t s, e;
    gate_group_range(G, gi, ng, s, e);
    uint32_t rlo = 0, rhi = 0xFFFFFFFFu;
    if (g.regions) {
      pos_of(u0);
      pos_of(u1);
      const int64_t d0 = jobs[j0 + u0].diag, d1 = jobs[j0 + u1].diag;
      const int64_t a0 = i64max(pqs[u0] + d0, 0), b0 = i64max(pqe[u0] + d0, 0);
      const int64_t a1 = i64max(pqs[u1] + d1, 0), b1 = i64max(pqe[u1] + d1, 0);
      rlo = static_cast<uint32_t>(i64min(a0, a1));
      rhi = static_cast<uint32_t>(i64max(b0, b1));
    }
    const GateJob jb = jobs[j0];
    cand[gi] = GateCandidate{jb.query, jb.target, e - s, total, static_cast<int64_t>(jobs[j0 + bi].diag), rlo, rhi};
    flag[gi] = 1;
  }
  gate_flush(&st->chains_used, n_chained);
}

// Rank keys of the kept candidates (sel: their group slots, in (query, target)
// order): (query, 2^31 - 1 - score) and the slot.
__global__ void __launch_bounds__(256) gate_rank_keys_kernel(const GateCandidate* cand, const uint32_t* sel,
                                                             const uint32_t* n_cand, uint64_t* keys, uint32_t* idx) {
  const uint32_t n = *n_cand;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t j = sel[i];
    const GateCandidate c = cand[j];
    keys[i] = (static_cast<uint64_t>(c.query) << 31) | static_cast<uint64_t>(0x7FFFFFFF - c.diag_score);
    idx[i] = j;
  }
}

// First and last rank position of every query in the ranked list.
__global__ void __launch_bounds__(256) gate_query_bounds_kernel(const uint64_t* keys, const uint32_t* n_cand,
                                                                uint32_t* qfirst, uint32_t* qcount) {
  const uint32_t n = *n_cand;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t q = static_cast<uint32_t>(keys[i] >> 31);
    if (i == 0 || static_cast<uint32_t>(keys[i - 1] >> 31) != q) qfirst[q] = i;
    if (i + 1 == n || static_cast<uint32_t>(keys[i + 1] >> 31) != q) qcount[q] = i + 1;  // end, made a count below
  }
}

// kept[q] = min(count, max_cand) for every query id (qcount holds the end).
__global__ void __launch_bounds__(256) gate_query_kept_kernel(const uint32_t* qfirst, const uint32_t* qend,
                                                              uint32_t n_prof, uint32_t max_cand, uint32_t* kept) {
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q <= n_prof; q += gridDim.x * blockDim.x) {
    uint32_t c = 0;
    if (q < n_prof) {
      c = qend[q] - qfirst[q];
      if (max_cand && c > max_cand) c = max_cand;
    }
    kept[q] = c;
  }
}

// out[pos] = the candidate of rank position i, pos = i without a cap, else the
// query's output offset + its rank inside the query (rank < max_cand).
__global__ void __launch_bounds__(256) gate_gather_kernel(const GateCandidate* cand, const uint64_t* keys,
                                                          const uint32_t* idx, const uint32_t* n_cand,
                                                          uint32_t max_cand, const uint32_t* qfirst,
                                                          const uint32_t* koff, GateCandidate* out) {
  const uint32_t n = *n_cand;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (max_cand == 0) {
      out[i] = cand[idx[i]];
    } else {
      const uint32_t q = static_cast<uint32_t>(keys[i] >> 31);
      const uint32_t r = i - qfirst[q];
      if (r < max_cand) out[koff[q] + r] = cand[idx[i]];
    }
  }
}

// Final counters: diagonals scored, candidates kept and cut.
__global__ void gate_finish_kernel(const uint32_t* n_groups, const uint32_t* joff, const uint32_t* n_cand,
                                   const uint32_t* koff, uint32_t n_prof, uint32_t max_cand, GateStats* st,
                                   unsigned long long* n_out) {
  const uint32_t nj = joff[*n_groups];
  const uint32_t nc = *n_cand;
  const uint32_t kept = max_cand ? koff[n_prof] : nc;
  st->diagonals_scored += nj;
  st->candidates += kept;
  st->candidates_capped += nc - kept;
  *n_out = kept;
}

}  // namespace st
