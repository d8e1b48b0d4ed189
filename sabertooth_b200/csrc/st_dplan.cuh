// Device-side planning of a batch of (profile, target) pairs for the packed
// 16-bit kernel: the same plan the host planner builds (pairs grouped by
// query, targets longest first, a tile class per query from the class rates,
// warp tasks of 64/G targets, CTA tasks capped at one CTA's share of their
// class, CTA tasks longest first), built on the GPU so that a large batch
// needs no host pass over its pairs beyond validation.
//
// Stages (one stream, in order):
//   classify   pair -> route (empty / 16-bit / 32-bit), SoA copies for the
//              32-bit kernel, a sort key (query, target length descending)
//   sort       radix sort of the keys (stable: equal keys keep pair order)
//   pick       per query: tile class by estimated time, warp-task count,
//              per-class totals (atomics)
//   split      per query: CTA-task count under the class's cost cap
//   order      queries sorted by class, exclusive scans of slots, warp tasks
//              and CTA tasks in that order (class segments are contiguous)
//   -- the host reads the per-class totals once, then sizes the rest --
//   emit       per query: slot records, warp tasks, CTA tasks + LPT keys
//   lpt        radix sort of CTA tasks by (class, cost descending), gather
#pragma once
#include <cstdint>

#include "../../include/sabertooth_b200.h"
#include "st_common.cuh"
#include "st_sw16.cuh"

namespace st {

constexpr int kDpMaxClasses = 32;
constexpr uint32_t kDpNoClass = 63;  // sort key of a query with no 16-bit pairs

struct DpClass {
  uint32_t G, R, C, W;
  uint32_t rows;      // G * R
  uint32_t S;         // targets per warp task, 64 / G
  uint32_t max_mpad;  // the largest staged row count that fits the class's shared memory
  float rate;         // streamed cells per second / 1e12 (0: not considered)
};

struct DpClasses {
  DpClass c[kDpMaxClasses];
  int n;
  int table[10][8];  // forced class per (query-length bin, mean target-length bin), -1: none
  uint32_t sms;      // SMs of the device (CTA-task cap: one CTA's share on two CTAs per SM)
};

// Per-class totals, filled by pick and split with atomics, read by the host.
struct DpTotals {
  uint32_t n_query[kDpMaxClasses];
  uint32_t n_wt[kDpMaxClasses];
  uint32_t n_cta[kDpMaxClasses];
  uint32_t max_mpad[kDpMaxClasses];
  uint32_t max_cols[kDpMaxClasses];        // widest warp task
  uint32_t max_cols_multi[kDpMaxClasses];  // widest warp task of a query with several passes
  unsigned long long cost[kDpMaxClasses];  // sum of warp-task costs (the CTA-task cap)
};

struct DpIn {
  const st_pair* pairs;
  uint32_t n;
  DeviceDb db;
  DeviceProfiles prof;
  uint32_t n_prof;
  uint32_t max_m16;  // longest query the 16-bit classes stage; longer ones take the 32-bit kernel
  uint32_t g16;      // gap costs inside the 16-bit kernel's range
  uint32_t tbits;    // bits of the sort key's target-length field
};

struct DpWork {
  // per pair
  uint32_t *pq, *pt;
  int32_t *pc, *pr;
  unsigned long long *keys, *keys_alt;
  uint32_t *vals, *vals_alt;  // after the sort: vals_sorted = pair ids grouped by query
  const uint32_t* vals_sorted;
  uint32_t* list32;      // 32-bit list (static entries first, 16-bit overflows appended by the kernels)
  uint32_t* list_count;  // device count of list32
  // per query
  uint32_t *qcnt, *qstart;  // 16-bit pairs per query and their start in vals_sorted
  uint32_t *qclass, *nwt, *ncta;
  uint32_t *qkey, *qkey_alt, *qid, *qid_alt;  // queries sorted by class
  const uint32_t* qid_sorted;
  uint32_t *a_slots, *a_wt, *a_cta;  // counts in class order, then their exclusive scans
  uint32_t *o_slots, *o_wt, *o_cta;
  DpTotals* totals;
};

struct DpOut {
  Sw16Slot* slots;
  Sw16WarpTask* wt;
  Sw16CtaTask* cta_raw;
  Sw16CtaTask* cta;  // LPT order, class segments in class order
  unsigned long long *cta_key, *cta_key_alt;
  uint32_t *cta_idx, *cta_idx_alt;
  const uint32_t* cta_idx_sorted;
  uint32_t n_cta;
};

__device__ __forceinline__ uint32_t dp_up4(uint32_t x) { return (x + 3u) & ~3u; }
__device__ __forceinline__ uint32_t dp_up16(uint32_t x) { return (x + 15u) & ~15u; }

__device__ __forceinline__ int dp_mbin(uint32_t m) {
  int b = 0;
  uint32_t lim = 32;
  while (b < 9 && m > lim) {
    ++b;
    lim <<= 1;
  }
  return b;
}
__device__ __forceinline__ int dp_nbin(uint32_t n) {
  int b = 0;
  uint32_t lim = 64;
  while (b < 7 && n > lim) {
    ++b;
    lim <<= 1;
  }
  return b;
}

// Shape of query m in class k.
struct DpShape {
  uint32_t P, mpad, minc, step_cost;
};
__device__ __forceinline__ DpShape dp_shape(const DpClass& k, uint32_t m) {
  DpShape s;
  s.P = (m + k.rows - 1) / k.rows;
  s.mpad = s.P * k.rows;
  s.minc = s.P > 1 ? max(32u, dp_up16(k.C * k.G)) : 32u;
  s.step_cost = k.R * k.C + 8;
  return s;
}

__device__ __forceinline__ unsigned long long dp_warp_sum(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}

// ---- classify: one thread per pair ----
__global__ void __launch_bounds__(256) dp_classify_kernel(const DpIn in, const DpWork w) {
  const unsigned long long sentinel = (in.tbits + 32 >= 64) ? ~0ull : ((1ull << (in.tbits + 32)) - 1);
  const uint32_t tmask = (in.tbits >= 32) ? 0xFFFFFFFFu : ((1u << in.tbits) - 1);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < in.n; i += gridDim.x * blockDim.x) {
    const uint4 x = __ldg(reinterpret_cast<const uint4*>(in.pairs) + i);
    const uint32_t q = x.x, t = x.y;
    const int32_t radius = static_cast<int32_t>(x.w);
    w.pq[i] = q;
    w.pt[i] = t;
    w.pc[i] = static_cast<int32_t>(x.z);
    w.pr[i] = radius;
    const uint32_t m = in.prof.qlen[q];
    const uint32_t tl = in.db.length[t];
    unsigned long long key = sentinel;
    if (m != 0 && tl != 0) {
      if (radius < 0 && in.g16 && in.prof.fits8[q] && m <= in.max_m16) {
        key = (static_cast<unsigned long long>(q) << in.tbits) | (tmask - tl);
        atomicAdd(&w.qcnt[q], 1u);
      } else {
        w.list32[atomicAdd(w.list_count, 1u)] = i;
      }
    }
    w.keys[i] = key;
    w.vals[i] = i;
  }
}

// ---- 32-bit list order: longest first by the steps a warp spends on a pair ----
// passes x (streamed columns + ramp); a banded pair streams one 256-row pass's band window per pass.  The
// key is inverted so that an ascending sort puts the costliest first.
__global__ void __launch_bounds__(256) dp_list_keys_kernel(const DpIn in, const DpWork w, uint32_t n_list,
                                                            unsigned long long* keys, uint32_t* vals) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_list; k += gridDim.x * blockDim.x) {
    const uint32_t i = w.list32[k];
    const unsigned long long m = in.prof.qlen[w.pq[i]], tl = in.db.length[w.pt[i]];
    const unsigned long long P = (m + 255) / 256;
    unsigned long long wc = tl;
    if (w.pr[i] >= 0) wc = min(tl, 256ull + 2ull * static_cast<unsigned long long>(w.pr[i]));
    const unsigned long long cost = min(P * (wc + 31), (1ull << 48) - 1);
    keys[k] = ((1ull << 48) - 1) - cost;
    vals[k] = i;
  }
}

// ---- pick: one warp per query ----
__global__ void __launch_bounds__(256) dp_pick_kernel(const DpIn in, const DpWork w, const DpClasses cls) {
  const uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (q >= in.n_prof) return;
  const uint32_t np = w.qcnt[q];
  if (lane == 0) {
    w.qid[q] = q;
    w.qkey[q] = kDpNoClass;
    w.qclass[q] = kDpNoClass;
    w.nwt[q] = 0;
  }
  if (np == 0) return;
  const uint32_t* v = w.vals_sorted + w.qstart[q];
  auto tl_at = [&](uint32_t j) { return in.db.length[w.pt[v[j]]]; };
  unsigned long long sum = 0;
  for (uint32_t j = lane; j < np; j += 32) sum += tl_at(j);
  sum = dp_warp_sum(sum);
  const uint32_t m = in.prof.qlen[q];
  const uint32_t mean_n = static_cast<uint32_t>(sum / np);
  int best = -1;
  const int forced = cls.table[dp_mbin(m)][dp_nbin(mean_n)];
  if (forced >= 0 && forced < cls.n && dp_shape(cls.c[forced], m).mpad <= cls.c[forced].max_mpad) best = forced;
  // least streamed cells / rate over the classes with a rate; if none of them
  // stages this query, least streamed cells over every class that does
  for (int pass = 0; pass < 2 && best < 0; ++pass) {
    double bt = 1e300;
    for (int k = 0; k < cls.n; ++k) {
      const DpClass& c = cls.c[k];
      if (pass == 0 && !(c.rate > 0.0f)) continue;
      const DpShape sh = dp_shape(c, m);
      if (sh.mpad > c.max_mpad) continue;
      const uint32_t nw = (np + c.S - 1) / c.S;
      unsigned long long cols = 0;
      for (uint32_t x = lane; x < nw; x += 32) cols += max(sh.minc, dp_up4(tl_at(x * c.S)));
      cols = dp_warp_sum(cols);
      const double t = static_cast<double>(cols) * c.S * sh.mpad / (pass == 0 ? c.rate : 1.0f);
      if (t < bt) {
        bt = t;
        best = k;
      }
    }
  }
  if (best < 0) return;  // cannot happen: the 16-bit route admits only queries some class stages
  const DpClass& c = cls.c[best];
  const DpShape sh = dp_shape(c, m);
  const uint32_t nw = (np + c.S - 1) / c.S;
  unsigned long long cost = 0;
  for (uint32_t x = lane; x < nw; x += 32) {
    const uint32_t nc = max(sh.minc, dp_up4(tl_at(x * c.S)));
    cost += static_cast<unsigned long long>(sh.P) * (nc / c.C) * sh.step_cost;
  }
  cost = dp_warp_sum(cost);
  if (lane == 0) {
    w.qclass[q] = static_cast<uint32_t>(best);
    w.qkey[q] = static_cast<uint32_t>(best);
    w.nwt[q] = nw;
    const uint32_t nc0 = max(sh.minc, dp_up4(tl_at(0)));
    atomicAdd(&w.totals->n_query[best], 1u);
    atomicAdd(&w.totals->n_wt[best], nw);
    atomicAdd(&w.totals->cost[best], cost);
    atomicMax(&w.totals->max_mpad[best], sh.mpad);
    atomicMax(&w.totals->max_cols[best], nc0);
    if (sh.P > 1) atomicMax(&w.totals->max_cols_multi[best], nc0);
  }
}

// CTA tasks of one query: consecutive warp tasks; a task ends at 128 warp
// tasks or, once it holds W of them, when its cost would pass the cap.
// f(w0, w1, cost) for each, in order.
template <class F>
__device__ __forceinline__ void dp_for_each_cta(const DpClass& c, const DpShape& sh, uint32_t nw,
                                                const uint32_t* v, const uint32_t* pt, const uint32_t* len,
                                                unsigned long long cap, F&& f) {
  uint32_t w0 = 0;
  unsigned long long acc = 0;
  for (uint32_t x = 0; x < nw; ++x) {
    const uint32_t nc = max(sh.minc, dp_up4(len[pt[v[x * c.S]]]));
    const unsigned long long cw = static_cast<unsigned long long>(sh.P) * (nc / c.C) * sh.step_cost;
    const uint32_t cnt = x - w0;
    if (cnt == 128u || (cnt >= c.W && acc + cw > cap)) {
      f(w0, x, acc);
      w0 = x;
      acc = 0;
    }
    acc += cw;
  }
  if (nw > w0) f(w0, nw, acc);
}

__device__ __forceinline__ unsigned long long dp_cap(const DpClasses& cls, const DpTotals* t, uint32_t k) {
  const unsigned long long cap = t->cost[k] / (2ull * cls.sms);
  return cap ? cap : 1ull;
}

// ---- split: one thread per query ----
__global__ void __launch_bounds__(256) dp_split_kernel(const DpIn in, const DpWork w, const DpClasses cls) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= in.n_prof) return;
  const uint32_t k = w.qclass[q];
  if (k == kDpNoClass) {
    w.ncta[q] = 0;
    return;
  }
  const DpClass& c = cls.c[k];
  const DpShape sh = dp_shape(c, in.prof.qlen[q]);
  uint32_t n = 0;
  dp_for_each_cta(c, sh, w.nwt[q], w.vals_sorted + w.qstart[q], w.pt, in.db.length, dp_cap(cls, w.totals, k),
                  [&](uint32_t, uint32_t, unsigned long long) { ++n; });
  w.ncta[q] = n;
  atomicAdd(&w.totals->n_cta[k], n);
}

// ---- counts in class order (one thread per position of the class-sorted queries) ----
__global__ void __launch_bounds__(256) dp_counts_kernel(const DpIn in, const DpWork w, const DpClasses cls) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > in.n_prof) return;
  if (i == in.n_prof) {  // the scans run over n_prof + 1 entries: the last gives the totals
    w.a_slots[i] = 0;
    w.a_wt[i] = 0;
    w.a_cta[i] = 0;
    return;
  }
  const uint32_t q = w.qid_sorted[i];
  const uint32_t k = w.qclass[q];
  const bool has = k != kDpNoClass;
  w.a_slots[i] = has ? w.nwt[q] * cls.c[k].S : 0u;
  w.a_wt[i] = has ? w.nwt[q] : 0u;
  w.a_cta[i] = has ? w.ncta[q] : 0u;
}

// ---- emit: one warp per position of the class-sorted queries ----
__global__ void __launch_bounds__(256) dp_emit_kernel(const DpIn in, const DpWork w, const DpClasses cls,
                                                      const DpOut out) {
  const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= in.n_prof) return;
  const uint32_t q = w.qid_sorted[i];
  const uint32_t k = w.qclass[q];
  if (k == kDpNoClass) return;
  const DpClass& c = cls.c[k];
  const uint32_t np = w.qcnt[q];
  const DpShape sh = dp_shape(c, in.prof.qlen[q]);
  const uint32_t nw = w.nwt[q];
  const uint32_t* v = w.vals_sorted + w.qstart[q];
  const uint32_t o_slot = w.o_slots[i], o_wt = w.o_wt[i], o_cta = w.o_cta[i];
  for (uint32_t x = lane; x < nw; x += 32) {
    const uint32_t sb = o_slot + x * c.S;
    uint32_t ncols = sh.minc;
    for (uint32_t s = 0; s < c.S; ++s) {
      const uint32_t j = x * c.S + s;
      Sw16Slot sl{kNoPair, 0, 0, 0};
      if (j < np) {
        const uint32_t pi = v[j];
        const uint32_t t = w.pt[pi];
        const uint32_t tl = in.db.length[t];
        sl.pair = pi;
        sl.toff16 = static_cast<uint32_t>(in.db.offset[t] / 16);
        sl.tlen16 = dp_up16(tl);
        sl.tlen = tl;
        ncols = max(ncols, dp_up4(tl));
      }
      out.slots[sb + s] = sl;
    }
    out.wt[o_wt + x] = Sw16WarpTask{sb, ncols};
  }
  if (lane == 0) {
    uint32_t t = o_cta;
    const unsigned long long kmask = (1ull << 44) - 1;
    dp_for_each_cta(c, sh, nw, v, w.pt, in.db.length, dp_cap(cls, w.totals, k),
                    [&](uint32_t w0, uint32_t w1, unsigned long long cost) {
                      out.cta_raw[t] = Sw16CtaTask{q, o_wt + w0, o_wt + w1, sh.mpad};
                      out.cta_key[t] = (static_cast<unsigned long long>(k) << 44) | (kmask - min(cost, kmask));
                      out.cta_idx[t] = t;
                      ++t;
                    });
  }
}

__global__ void __launch_bounds__(256) dp_gather_cta_kernel(const DpOut out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < out.n_cta) out.cta[i] = out.cta_raw[out.cta_idx_sorted[i]];
}

__global__ void __launch_bounds__(256) dp_iota_kernel(uint32_t* v, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

__global__ void __launch_bounds__(256) dp_fill_zline_kernel(uint2* z, uint32_t n, uint32_t v) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = make_uint2(0u, v);
}

}  // namespace st
