// Seed hits on the device: the seed stage of the reference's prefilter_query
// (src/prefilter.rs:816-995) over a device-resident seed index.
//
// Index (SeedIndex, src/index.rs:1059-1074 window_ok): every window of every
// database sequence whose care positions (the seed pattern's '1's) hold codes
// < 20, keyed by code = care residues in base 20; a direct table of 20^w + 1
// offsets (w <= 7) over (sequence, window start) postings, filled by one warp
// per sequence with one atomic counter per code (the order inside a code does
// not matter: hits are grouped by a sort later).
//
// Queries, one thread per window (query, start):
//   count  eligibility (no care residue >= 20 for sequence queries), the number
//          of k-mers over the 20 standard residues scoring >= kmer_score from a
//          histogram of partial sums pruned at the threshold (the counting pass
//          of cap_boundary, :571-609), and, above the cap, the boundary score t*
//          and how many ties at t* are kept;
//   emit   the window's k-mers by a depth-first walk in rank-lexicographic order
//          with exact suffix-maximum pruning (top_kmers, :470-568): every k-mer
//          above t* (or >= the threshold when not capped) and the first ties at
//          t* in that order — the first `cap` k-mers of the canonical order;
//          the query's own k-mer is added when it is not among them (exact seeds);
//   posts  each k-mer's posting count (skipped above max_seed_occ, push_seed
//          :853-869), then one hit (query, target, tpos - qpos, qpos) per posting.
#pragma once
#include "st_common.cuh"
#include "st_gate.cuh"

namespace st {

constexpr int kSeedMaxW = 7;        // direct table: 20^7 + 1 offsets
constexpr int kSeedAA = 20;         // standard residues
constexpr int kSeedMaxBins = 1024;  // partial-sum histogram width (score range of a window above the threshold)
constexpr uint32_t kSeedNone = 0xFFFFFFFFu;

struct SeedPat {
  uint32_t w;
  uint32_t span;
  uint32_t offs[12];
};

struct SeedPost {
  uint32_t target;
  uint32_t tpos;
};

// A query position's 20 standard residues by score descending, residue
// ascending (sorted_row, src/prefilter.rs:433-441).
struct SeedRow {
  int32_t sc[kSeedAA];
  uint8_t res[kSeedAA];
};

struct SeedWin {  // per window: boundary of the kept set
  int32_t tstar;  // INT32_MIN: not capped
  uint32_t need;  // ties at t* kept
};

struct SeedSeed {
  uint32_t code;  // kSeedNone: an unused exact-seed slot
  uint32_t window;
};

struct SeedStatsDev {  // the layout of st_seed_stats
  unsigned long long windows, windows_skipped, kmers_generated, windows_at_cap, exact_seeds_added, seeds,
      postings_visited, seeds_over_occ_cap, postings_skipped_occ, errors;
};

__device__ __forceinline__ bool seed_window_code(const uint8_t* s, const SeedPat& p, uint32_t& code) {
  uint32_t c = 0;
  for (uint32_t i = 0; i < p.w; ++i) {
    const uint32_t r = s[p.offs[i]];
    if (r >= kSeedAA) return false;
    c = c * kSeedAA + r;
  }
  code = c;
  return true;
}

// One warp per sequence, lanes over its window starts.
template <bool FILL>
__global__ void __launch_bounds__(256) seed_index_kernel(DeviceDb db, SeedPat p, uint32_t* cnt, SeedPost* post) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  for (uint32_t s = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; s < db.n_seqs; s += warps) {
    const uint32_t n = db.length[s];
    if (n < p.span) continue;
    const uint8_t* t = db.arena + db.offset[s];
    for (uint32_t st = lane; st + p.span <= n; st += 32) {
      uint32_t code;
      if (!seed_window_code(t + st, p, code)) continue;
      if (FILL)
        post[atomicAdd(&cnt[code], 1u)] = SeedPost{s, st};
      else
        atomicAdd(&cnt[code], 1u);
    }
  }
}

__global__ void __launch_bounds__(128) seed_sort_rows_kernel(DeviceProfiles prof, const uint32_t* qids,
                                                             const uint32_t* row0, SeedRow* rows) {
  const uint32_t qi = blockIdx.x;
  const uint32_t q = qids[qi];
  const uint32_t m = prof.qlen[q];
  const int32_t* p32 = prof.p32[q];
  const uint32_t s32 = prof.stride32[q];
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
    SeedRow r;
    for (int a = 0; a < kSeedAA; ++a) {
      r.sc[a] = p32[a * s32 + i];
      r.res[a] = static_cast<uint8_t>(a);
    }
    for (int a = 1; a < kSeedAA; ++a)  // stable: equal scores keep residue order
      for (int b = a; b > 0 && r.sc[b] > r.sc[b - 1]; --b) {
        const int32_t ts = r.sc[b];
        r.sc[b] = r.sc[b - 1];
        r.sc[b - 1] = ts;
        const uint8_t tr = r.res[b];
        r.res[b] = r.res[b - 1];
        r.res[b - 1] = tr;
      }
    rows[row0[qi] + i] = r;
  }
}

struct SeedQ {
  const uint32_t* qids;
  const uint32_t* woff;  // first window of each query, n_q + 1 entries
  const uint32_t* row0;  // first sorted row of each query
  const uint8_t* res;    // residues of sequence queries (NULL: profile queries)
  const SeedRow* rows;
  uint32_t n_q;
  uint32_t n_win;
  int32_t thr;
  uint32_t cap;
  uint32_t exact;  // add the query's own k-mer
};

__device__ __forceinline__ void seed_window_of(const SeedQ& Q, uint32_t wi, uint32_t& qi, uint32_t& start) {
  uint32_t lo = 0, hi = Q.n_q;  // last qi with woff[qi] <= wi
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (Q.woff[mid] <= wi) lo = mid; else hi = mid;
  }
  qi = lo;
  start = wi - Q.woff[lo];
}

// Eligibility, exact code and the window's sorted rows (pointers into Q.rows).
__device__ __forceinline__ bool seed_window_rows(const SeedQ& Q, const SeedPat& P, uint32_t qi, uint32_t start,
                                                 const SeedRow** wr, uint32_t& exact) {
  const uint32_t base = Q.row0[qi] + start;
  uint32_t e = 0;
  for (uint32_t i = 0; i < P.w; ++i) {
    if (Q.res) {
      const uint32_t r = Q.res[base + P.offs[i]];
      if (r >= kSeedAA) return false;
      e = e * kSeedAA + r;
    }
    wr[i] = Q.rows + base + P.offs[i];
  }
  exact = e;
  return true;
}

__global__ void __launch_bounds__(128) seed_count_kernel(SeedQ Q, SeedPat P, uint32_t* slots, SeedWin* win,
                                                         SeedStatsDev* st) {
  unsigned long long n_skip = 0, n_cap = 0, n_err = 0;
  uint32_t dist[kSeedMaxBins], tmp[kSeedMaxBins];
  for (uint32_t wi = blockIdx.x * blockDim.x + threadIdx.x; wi <= Q.n_win; wi += gridDim.x * blockDim.x) {
    uint32_t n_slots = 0;
    if (wi < Q.n_win) {
      uint32_t qi, start, exact;
      seed_window_of(Q, wi, qi, start);
      const SeedRow* wr[kSeedMaxW];
      SeedWin wv{INT32_MIN, 0};
      if (!seed_window_rows(Q, P, qi, start, wr, exact)) {
        ++n_skip;
      } else {
        int32_t smax[kSeedMaxW + 1];
        smax[P.w] = 0;
        for (int i = static_cast<int>(P.w) - 1; i >= 0; --i) smax[i] = smax[i + 1] + wr[i]->sc[0];
        uint32_t count = 0;
        if (smax[0] >= Q.thr && Q.cap > 0) {
          // histogram of the partial sums that can still reach the threshold
          int32_t lo = 0, hi = 0;
          dist[0] = 1;
          bool ok = true;
          for (uint32_t i = 0; i < P.w && ok; ++i) {
            const int32_t nhi = hi + wr[i]->sc[0];
            const int32_t nlo = max(lo + wr[i]->sc[kSeedAA - 1], Q.thr - smax[i + 1]);
            if (nhi - nlo + 1 > kSeedMaxBins) {
              ok = false;
              break;
            }
            for (int32_t b = 0; b <= nhi - nlo; ++b) tmp[b] = 0;
            for (int32_t off = 0; off <= hi - lo; ++off) {
              const uint32_t cnt = dist[off];
              if (!cnt) continue;
              const int32_t s = lo + off;
              for (int a = 0; a < kSeedAA; ++a) {
                const int32_t t = s + wr[i]->sc[a];
                if (t < nlo) break;
                tmp[t - nlo] += cnt;
              }
            }
            for (int32_t b = 0; b <= nhi - nlo; ++b) dist[b] = tmp[b];
            lo = nlo;
            hi = nhi;
          }
          if (!ok) {
            ++n_err;
          } else {
            for (int32_t b = 0; b <= hi - lo; ++b) count += dist[b];
            if (count > Q.cap) {
              uint32_t above = 0;
              int32_t t = hi;
              for (; t > lo; --t) {
                const uint32_t cnt = dist[t - lo];
                if (above + cnt >= Q.cap) break;
                above += cnt;
              }
              wv.tstar = t;
              wv.need = Q.cap - above;
              count = Q.cap;
              ++n_cap;
            }
          }
        }
        n_slots = count + (Q.exact ? 1u : 0u);
      }
      win[wi] = wv;
    }
    slots[wi] = n_slots;
  }
  gate_flush(&st->windows_skipped, n_skip);
  gate_flush(&st->windows_at_cap, n_cap);
  gate_flush(&st->errors, n_err);
}

// The kept k-mers of each window in rank-lexicographic depth-first order.
__global__ void __launch_bounds__(128) seed_emit_kernel(SeedQ Q, SeedPat P, const uint32_t* soff, const SeedWin* win,
                                                        SeedSeed* seeds, SeedStatsDev* st) {
  unsigned long long n_gen = 0, n_exact = 0, n_err = 0;
  for (uint32_t wi = blockIdx.x * blockDim.x + threadIdx.x; wi < Q.n_win; wi += gridDim.x * blockDim.x) {
    const uint32_t o0 = soff[wi], o1 = soff[wi + 1];
    if (o1 == o0) continue;
    uint32_t qi, start, exact;
    seed_window_of(Q, wi, qi, start);
    const SeedRow* wr[kSeedMaxW];
    seed_window_rows(Q, P, qi, start, wr, exact);
    const SeedWin wv = win[wi];
    const uint32_t w = P.w, last = w - 1;
    int32_t smax[kSeedMaxW + 1];
    smax[w] = 0;
    for (int i = static_cast<int>(w) - 1; i >= 0; --i) smax[i] = smax[i + 1] + wr[i]->sc[0];
    const bool capped = wv.tstar != INT32_MIN;
    int32_t thr = capped ? (wv.need ? wv.tstar : wv.tstar + 1) : Q.thr;
    uint32_t ties = wv.need;
    uint32_t n = 0;
    bool have_exact = false;
    const uint32_t n_kmers = o1 - o0 - (Q.exact ? 1u : 0u);
    if (n_kmers > 0) {
      uint32_t rank[kSeedMaxW], code[kSeedMaxW + 1];
      int32_t part[kSeedMaxW + 1];
      part[0] = 0;
      code[0] = 0;
      rank[0] = 0;
      uint32_t d = 0;
      for (;;) {
        if (d == last) {
          const int32_t bs = part[last];
          const uint32_t bc = code[last] * kSeedAA;
          for (int a = 0; a < kSeedAA; ++a) {
            const int32_t ns = bs + wr[last]->sc[a];
            if (ns < thr) break;
            const uint32_t cc = bc + wr[last]->res[a];
            if (n < n_kmers) seeds[o0 + n] = SeedSeed{cc, wi};  // n == n_kmers at the end (checked below)
            ++n;
            have_exact |= cc == exact;
            if (capped && ns == wv.tstar && --ties == 0) thr = wv.tstar + 1;
          }
          if (last == 0) break;
          d = last - 1;
          ++rank[d];
          continue;
        }
        const uint32_t r = rank[d];
        if (r < kSeedAA) {
          const int32_t ns = part[d] + wr[d]->sc[r];
          if (ns + smax[d + 1] >= thr) {
            part[d + 1] = ns;
            code[d + 1] = code[d] * kSeedAA + wr[d]->res[r];
            ++d;
            rank[d] = 0;
            continue;
          }
        }
        if (d == 0) break;
        --d;
        ++rank[d];
      }
    }
    n_err += n != n_kmers;
    n_gen += n;
    if (Q.exact) {
      if (!have_exact) {
        seeds[o0 + n_kmers] = SeedSeed{exact, wi};
        ++n_exact;
        ++n_gen;
      } else {
        seeds[o0 + n_kmers] = SeedSeed{kSeedNone, wi};
      }
    }
  }
  gate_flush(&st->kmers_generated, n_gen);
  gate_flush(&st->exact_seeds_added, n_exact);
  gate_flush(&st->errors, n_err);
}

// Posting count of each seed (0 for an unused slot, an empty code, or a code
// above max_seed_occ); n_seeds + 1 entries, the last 0.
__global__ void __launch_bounds__(256) seed_post_count_kernel(const SeedSeed* seeds, uint32_t n_seeds,
                                                              const uint32_t* off, uint32_t occ_cap, uint32_t* cnt,
                                                              SeedStatsDev* st) {
  unsigned long long n_seed = 0, n_post = 0, n_over = 0, n_skip = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n_seeds; i += gridDim.x * blockDim.x) {
    uint32_t len = 0;
    if (i < n_seeds && seeds[i].code != kSeedNone) {
      const uint32_t c = seeds[i].code;
      len = off[c + 1] - off[c];
      if (len > 0 && occ_cap > 0 && len > occ_cap) {
        ++n_over;
        n_skip += len;
        len = 0;
      } else if (len > 0) {
        ++n_seed;
        n_post += len;
      }
    }
    cnt[i] = len;
  }
  gate_flush(&st->seeds, n_seed);
  gate_flush(&st->postings_visited, n_post);
  gate_flush(&st->seeds_over_occ_cap, n_over);
  gate_flush(&st->postings_skipped_occ, n_skip);
}

// One hit per posting.  A warp takes 32 consecutive seeds, whose hits are one
// contiguous range of the output; lane k writes output positions k, k + 32, ...
// and finds the seed of each by a binary search over the 32 seeds' offsets held
// in the lanes, so reads of the postings and writes of the hits are coalesced
// whatever the list lengths.
__global__ void __launch_bounds__(256) seed_hits_kernel(SeedQ Q, const SeedSeed* seeds, uint32_t n_seeds,
                                                        const uint32_t* cnt, const uint32_t* hoff, const uint32_t* off,
                                                        const SeedPost* post, GateSeedHit* hits) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n_groups = (n_seeds + 31) / 32;
  for (uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) / 32; g < n_groups; g += (gridDim.x * blockDim.x) / 32) {
    const uint32_t s = g * 32 + lane;
    // this lane's seed: first output position, posting start, query and position
    uint32_t o = 0, pstart = 0, q = 0, start = 0;
    if (s < n_seeds) {
      o = hoff[s];
      if (cnt[s]) {
        const SeedSeed sd = seeds[s];
        uint32_t qi;
        seed_window_of(Q, sd.window, qi, start);
        q = Q.qids[qi];
        pstart = off[sd.code];
      }
    }
    const uint32_t last = min(n_seeds, g * 32 + 32);
    const uint32_t o_begin = __shfl_sync(0xFFFFFFFFu, o, 0);
    const uint32_t o_end = hoff[last];
    for (uint32_t base = o_begin; base < o_end; base += 32) {  // every lane runs every round (shuffles)
      const uint32_t k = base + lane;
      const bool live = k < o_end;
      // last lane j with offset <= k (lanes past the group's seeds are never chosen)
      uint32_t j = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const uint32_t cand = j + step;
        const uint32_t oc = __shfl_sync(0xFFFFFFFFu, o, cand & 31);
        if (cand < last - g * 32 && oc <= k) j = cand;
      }
      const uint32_t oj = __shfl_sync(0xFFFFFFFFu, o, j);
      const uint32_t pj = __shfl_sync(0xFFFFFFFFu, pstart, j);
      const uint32_t qj = __shfl_sync(0xFFFFFFFFu, q, j);
      const uint32_t sj = __shfl_sync(0xFFFFFFFFu, start, j);
      if (live) {
        const SeedPost ps = post[pj + (k - oj)];
        hits[k] = GateSeedHit{qj, ps.target, static_cast<int32_t>(ps.tpos) - static_cast<int32_t>(sj), sj};
      }
    }
  }
}

}  // namespace st
