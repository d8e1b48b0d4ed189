// Serving loop: continuous batching of scoring requests on one context.
//
// A request is one query (its int32 [m][21] rows) and the database targets
// to score it against (optionally banded). Client threads submit requests at
// any time and wait for them by id. One worker thread forms batches from
// the requests that have arrived, in arrival order, up to a pair cap and a
// device-memory budget; it keeps two batches in flight: while one runs on
// the GPU the next is built (profiles uploaded, pairs filled) and launched,
// so requests that arrive during a batch join the next one and their work
// overlaps the running one on the device. Results are the same as scoring
// each request alone: every pair's score depends only on its own inputs.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/sabertooth_b200.h"

__attribute__((visibility("hidden"))) void st_internal_set_error(const char* msg);

namespace {

using Clock = std::chrono::steady_clock;

// With ST_TRACE set: worker steps slower than 5 ms go to stderr.
bool server_trace() {
  static const bool on = [] {
    const char* e = std::getenv("ST_TRACE");
    return e && *e && *e != '0';
  }();
  return on;
}
void trace_slow(const char* what, Clock::time_point t0, size_t reqs, size_t pairs) {
  if (!server_trace()) return;
  const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  if (ms > 5.0) fprintf(stderr, "[st] server %s %.3f ms (%zu requests, %zu pairs)\n", what, ms, reqs, pairs);
}

// Score rows of one submission: one request's, or a whole bulk submission's
// (its requests hold consecutive rows of the block).
struct RowBlock {
  std::vector<int32_t> rows;
};

struct Request {
  uint64_t id = 0;
  uint32_t m = 0;
  std::shared_ptr<RowBlock> block;  // rows [row0, row0 + m) of the block are this request's
  uint64_t row0 = 0;
  std::vector<st_pair> pairs;  // profile field filled when batched
  std::vector<int32_t> scores;
  Clock::time_point t_submit, t_done;
  bool done = false;
  int status = ST_OK;
  std::string error;
  uint64_t bytes = 0;  // device-memory estimate while in flight
};

struct Batch {
  std::vector<std::shared_ptr<Request>> reqs;
  std::vector<uint32_t> ids;  // profile ids
  std::vector<st_pair> pairs;
  std::vector<int32_t> scores;
  st_batch* handle = nullptr;
  uint64_t bytes = 0;
};

// Device bytes a request holds while in flight: its profile layouts (int8
// and int32, rounded as the library stores them) and per-pair plan buffers.
uint64_t request_bytes(uint32_t m, uint64_t n_pairs) {
  const uint64_t s8 = ((m + 15) / 16) * 16, s32 = std::max<uint64_t>(((m + 255) / 256) * 256, 256);
  return 22 * s8 + 22 * 4 * s32 + 4096 + n_pairs * 256;
}

}  // namespace

struct st_server {
  st_ctx* ctx = nullptr;
  int32_t open = 0, ext = 0;
  uint64_t max_pairs = 0, budget = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> pending;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread worker;
  uint64_t batches = 0, batched_pairs = 0;
  int32_t* arena = nullptr;  // pinned rows of the batch being launched (uploaded before the next one fills it)
  size_t arena_bytes = 0;

  void run();
  void finish(std::unique_ptr<Batch>& b);
  int launch(std::unique_ptr<Batch>& b);
};

// Builds a batch's profiles and pairs and launches it; on failure every
// request of the batch completes with the error.
int st_server::launch(std::unique_ptr<Batch>& b) {
  std::vector<uint64_t> offs(b->reqs.size() + 1, 0);
  for (size_t i = 0; i < b->reqs.size(); ++i) offs[i + 1] = offs[i] + b->reqs[i]->m;
  size_t n_pairs = 0;
  for (size_t i = 0; i < b->reqs.size(); ++i) n_pairs += b->reqs[i]->pairs.size();
  b->ids.assign(b->reqs.size(), 0);
  // A batch that is one run of consecutive requests of a bulk submission uploads straight from the
  // submission's rows (the library stages them, copy and upload overlapped); any other batch is gathered
  // into the pinned arena first.
  bool run = true;
  for (size_t i = 1; i < b->reqs.size() && run; ++i)
    run = b->reqs[i]->block == b->reqs[0]->block && b->reqs[i]->row0 == b->reqs[i - 1]->row0 + b->reqs[i - 1]->m;
  int rc;
  if (run && offs.back() > 0) {
    rc = st_profiles_create(ctx, b->reqs[0]->block->rows.data() + b->reqs[0]->row0 * 21, offs.data(),
                            static_cast<uint32_t>(b->reqs.size()), b->ids.data());
  } else {
    const size_t need = std::max<size_t>(static_cast<size_t>(offs.back()) * 21 * 4, 64);
    if (arena_bytes < need) {
      // at least 16 MB, and at least double: freeing pinned memory waits for the
      // batch in flight, so growth should be rare
      const size_t want = std::max<size_t>({need + need / 4, 2 * arena_bytes, 16u << 20});
      if (arena) cudaFreeHost(arena);
      arena = nullptr;
      arena_bytes = 0;
      if (cudaHostAlloc(reinterpret_cast<void**>(&arena), want, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        st_internal_set_error("serving: pinned host allocation failed");
        return ST_ENOMEM;
      }
      arena_bytes = want;
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < static_cast<int64_t>(b->reqs.size()); ++i)
      if (b->reqs[i]->m)
        memcpy(arena + offs[i] * 21, b->reqs[i]->block->rows.data() + b->reqs[i]->row0 * 21,
               static_cast<size_t>(b->reqs[i]->m) * 21 * 4);
    rc = st_profiles_create(ctx, arena, offs.data(), static_cast<uint32_t>(b->reqs.size()), b->ids.data());
  }
  if (rc != ST_OK) return rc;
  b->pairs.reserve(n_pairs);
  for (size_t i = 0; i < b->reqs.size(); ++i)
    for (st_pair p : b->reqs[i]->pairs) {
      p.profile = b->ids[i];
      b->pairs.push_back(p);
    }
  b->scores.assign(n_pairs, 0);
  rc = st_sw_score_pairs_async(ctx, b->pairs.data(), n_pairs, open, ext, b->scores.data(), nullptr, &b->handle);
  if (rc != ST_OK) {
    st_profiles_free(ctx, b->ids.data(), static_cast<uint32_t>(b->ids.size()));
    b->ids.clear();
  }
  return rc;
}

void st_server::finish(std::unique_ptr<Batch>& b) {
  int rc = ST_OK;
  std::string err;
  if (b->handle) {
    rc = st_batch_wait(b->handle);
    if (rc != ST_OK) err = st_last_error();
  }
  if (!b->ids.empty()) st_profiles_free(ctx, b->ids.data(), static_cast<uint32_t>(b->ids.size()));
  const Clock::time_point now = Clock::now();
  std::lock_guard<std::mutex> lk(mu);
  size_t at = 0;
  for (auto& r : b->reqs) {
    r->scores.assign(b->scores.begin() + at, b->scores.begin() + at + r->pairs.size());
    at += r->pairs.size();
    r->status = rc;
    r->error = err;
    r->t_done = now;
    r->done = true;
  }
  ++batches;
  batched_pairs += at;
  cv_done.notify_all();
}

void st_server::run() {
  std::deque<std::unique_ptr<Batch>> inflight;
  uint64_t inflight_bytes = 0;
  for (;;) {
    std::unique_ptr<Batch> b;
    {
      std::unique_lock<std::mutex> lk(mu);
      if (inflight.empty()) {
        cv_work.wait(lk, [&] { return stop || !pending.empty(); });
      } else if (inflight.size() == 1 && pending.empty()) {
        // one batch running and nothing waiting: watch for arrivals and for the batch's end
        cv_work.wait_for(lk, std::chrono::microseconds(200), [&] { return stop || !pending.empty(); });
        if (pending.empty() && st_batch_query(inflight.front()->handle) == 1) continue;
      }
      if (stop && pending.empty() && inflight.empty()) return;
      if (inflight.size() < 2 && !pending.empty()) {
        // arrival order, up to the pair cap and the memory left beside the batches in flight
        b.reset(new Batch);
        uint64_t pairs = 0;
        while (!pending.empty()) {
          const auto& r = pending.front();
          const bool first = b->reqs.empty();
          if (!first && (pairs + r->pairs.size() > max_pairs || inflight_bytes + b->bytes + r->bytes > budget)) break;
          pairs += r->pairs.size();
          b->bytes += r->bytes;
          b->reqs.push_back(r);
          pending.pop_front();
        }
      }
    }
    if (b) {
      const Clock::time_point t0 = Clock::now();
      const int rc = launch(b);
      trace_slow("launch", t0, b->reqs.size(), b->pairs.size());
      if (rc != ST_OK) {
        b->handle = nullptr;
        const std::string err = st_last_error();
        std::lock_guard<std::mutex> lk(mu);
        for (auto& r : b->reqs) {
          r->status = rc;
          r->error = err;
          r->t_done = Clock::now();
          r->done = true;
        }
        cv_done.notify_all();
      } else {
        inflight_bytes += b->bytes;
        inflight.push_back(std::move(b));
      }
      // with one batch in flight, build the next at once if requests are waiting
      std::lock_guard<std::mutex> lk(mu);
      if (inflight.size() < 2 && !pending.empty()) continue;
    }
    if (!inflight.empty()) {
      inflight_bytes -= inflight.front()->bytes;
      const Clock::time_point t0 = Clock::now();
      const size_t nr = inflight.front()->reqs.size(), np = inflight.front()->pairs.size();
      finish(inflight.front());
      trace_slow("finish", t0, nr, np);
      inflight.pop_front();
    }
  }
}

extern "C" st_server* st_server_create(st_ctx* ctx, int32_t open, int32_t ext, uint64_t max_batch_pairs,
                                       uint64_t hbm_budget_bytes) {
  if (!ctx) {
    st_internal_set_error("st_server_create: null context");
    return nullptr;
  }
  auto s = std::make_unique<st_server>();
  s->ctx = ctx;
  s->open = open;
  s->ext = ext;
  // the pinned arena that gathers a batch's rows, allocated now rather than by the first batch that
  // gathers (a large pinned allocation stalls the worker for milliseconds)
  if (cudaHostAlloc(reinterpret_cast<void**>(&s->arena), 16u << 20, cudaHostAllocPortable) == cudaSuccess) {
    s->arena_bytes = 16u << 20;
  } else {
    cudaGetLastError();
    s->arena = nullptr;
  }
  s->max_pairs = max_batch_pairs ? max_batch_pairs : (1ull << 22);
  s->budget = hbm_budget_bytes ? hbm_budget_bytes : (16ull << 30);
  st_server* p = s.get();
  s->worker = std::thread([p] { p->run(); });
  return s.release();
}

extern "C" int st_server_submit(st_server* s, const int32_t* rows, uint32_t m, const uint32_t* targets,
                                const int32_t* band_center, const int32_t* band_radius, uint32_t n,
                                uint64_t* request_id) {
  if (!s || !request_id || (m && !rows) || (n && !targets)) {
    st_internal_set_error("st_server_submit: null argument");
    return ST_EINVAL;
  }
  auto r = std::make_shared<Request>();
  r->m = m;
  r->block = std::make_shared<RowBlock>();
  r->block->rows.assign(rows, rows + static_cast<size_t>(m) * 21);
  r->pairs.resize(n);
  for (uint32_t i = 0; i < n; ++i)
    r->pairs[i] = st_pair{0, targets[i], band_center ? band_center[i] : 0, band_radius ? band_radius[i] : -1};
  r->bytes = request_bytes(m, n);
  if (r->bytes > s->budget) {
    st_internal_set_error("st_server_submit: request needs more device memory than the server's budget");
    return ST_ENOMEM;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) {
    st_internal_set_error("st_server_submit: server is stopping");
    return ST_ESTATE;
  }
  r->id = s->next_id++;
  r->t_submit = Clock::now();
  s->live[r->id] = r;
  s->pending.push_back(r);
  *request_id = r->id;
  s->cv_work.notify_one();
  return ST_OK;
}

extern "C" int st_server_submit_many(st_server* s, uint32_t n_requests, const int32_t* rows, const uint64_t* row_offsets,
                                     const uint32_t* targets, const uint64_t* target_offsets, const int32_t* band_center,
                                     const int32_t* band_radius, uint64_t* request_ids) {
  if (!s || !request_ids || (n_requests && (!row_offsets || !target_offsets))) {
    st_internal_set_error("st_server_submit_many: null argument");
    return ST_EINVAL;
  }
  for (uint32_t k = 0; k < n_requests; ++k) {
    const uint64_t r0 = row_offsets[k], r1 = row_offsets[k + 1], t0 = target_offsets[k], t1 = target_offsets[k + 1];
    if (r1 < r0 || t1 < t0 || (r1 > r0 && !rows) || (t1 > t0 && !targets)) {
      st_internal_set_error("st_server_submit_many: bad offsets");
      return ST_EINVAL;
    }
    if (request_bytes(static_cast<uint32_t>(r1 - r0), t1 - t0) > s->budget) {
      st_internal_set_error("st_server_submit_many: a request needs more device memory than the server's budget");
      return ST_ENOMEM;
    }
  }
  std::vector<std::shared_ptr<Request>> rs(n_requests);
  // the submission's rows in one block (copied in parallel), each request a run of it
  auto block = std::make_shared<RowBlock>();
  const uint64_t first = n_requests ? row_offsets[0] : 0, last = n_requests ? row_offsets[n_requests] : 0;
  block->rows.resize((last - first) * 21);
  {
    const int64_t chunk = 1 << 20;  // values per copy task
    const int64_t total = static_cast<int64_t>(block->rows.size());
#pragma omp parallel for schedule(static)
    for (int64_t o = 0; o < total; o += chunk)
      memcpy(block->rows.data() + o, rows + first * 21 + o, static_cast<size_t>(std::min(chunk, total - o)) * 4);
  }
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t k = 0; k < static_cast<int64_t>(n_requests); ++k) {
    auto r = std::make_shared<Request>();
    const uint64_t r0 = row_offsets[k], r1 = row_offsets[k + 1], t0 = target_offsets[k], t1 = target_offsets[k + 1];
    r->m = static_cast<uint32_t>(r1 - r0);
    r->block = block;
    r->row0 = r0 - first;
    r->pairs.resize(t1 - t0);
    for (uint64_t i = t0; i < t1; ++i)
      r->pairs[i - t0] = st_pair{0, targets[i], band_center ? band_center[i] : 0, band_radius ? band_radius[i] : -1};
    r->bytes = request_bytes(r->m, t1 - t0);
    rs[k] = std::move(r);
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) {
    st_internal_set_error("st_server_submit_many: server is stopping");
    return ST_ESTATE;
  }
  const Clock::time_point now = Clock::now();
  for (uint32_t k = 0; k < n_requests; ++k) {
    rs[k]->id = s->next_id++;
    rs[k]->t_submit = now;
    s->live[rs[k]->id] = rs[k];
    s->pending.push_back(rs[k]);
    request_ids[k] = rs[k]->id;
  }
  s->cv_work.notify_one();
  return ST_OK;
}

extern "C" int st_server_wait(st_server* s, uint64_t request_id, int32_t* scores, uint32_t cap, double* latency_ms) {
  if (!s) {
    st_internal_set_error("st_server_wait: null server");
    return ST_EINVAL;
  }
  std::shared_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->live.find(request_id);
    if (it == s->live.end()) {
      st_internal_set_error("st_server_wait: unknown request id");
      return ST_EINVAL;
    }
    r = it->second;
    s->cv_done.wait(lk, [&] { return r->done; });
    s->live.erase(request_id);
  }
  if (r->status != ST_OK) {
    st_internal_set_error(r->error.c_str());
    return r->status;
  }
  if (scores) memcpy(scores, r->scores.data(), std::min<size_t>(cap, r->scores.size()) * 4);
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  return ST_OK;
}

extern "C" int st_server_stats(st_server* s, uint64_t* batches, uint64_t* pairs) {
  if (!s) {
    st_internal_set_error("st_server_stats: null server");
    return ST_EINVAL;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (batches) *batches = s->batches;
  if (pairs) *pairs = s->batched_pairs;
  return ST_OK;
}

extern "C" void st_server_destroy(st_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  if (s->arena) cudaFreeHost(s->arena);
  delete s;
}

// ---------------------------------------------------------------------------
// Search serving: requests are bare queries; each batch runs the whole search
// (profiles, seeds -> evidence -> chains -> gate on the device, then SW over
// every candidate).  One batch at a time (the prefilter's sizing reads share
// the context's stream with the scoring); requests that arrive during a batch
// form the next one.  A request's candidates and scores equal those of the
// query searched alone: every candidate depends only on its own query's hits.
// ---------------------------------------------------------------------------
namespace {

struct SearchRequest {
  uint64_t id = 0;
  uint32_t m = 0;
  std::vector<int32_t> rows;
  std::vector<uint8_t> residues;  // empty: a profile query
  std::vector<st_candidate> cands;
  std::vector<int32_t> scores;
  Clock::time_point t_submit, t_done;
  bool done = false;
  int status = ST_OK;
  std::string error;
};

}  // namespace

struct st_search_server {
  st_ctx* ctx = nullptr;
  st_seed_params sp{};
  st_prefilter_params gp{};
  uint32_t max_queries = 0;
  bool sequence = true;  // queries carry residues
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<SearchRequest>> pending;
  std::unordered_map<uint64_t, std::shared_ptr<SearchRequest>> live;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread worker;
  uint64_t batches = 0, queries = 0;
  void run();
  int search(std::vector<std::shared_ptr<SearchRequest>>& b);
};

int st_search_server::search(std::vector<std::shared_ptr<SearchRequest>>& b) {
  const size_t n = b.size();
  std::vector<uint64_t> offs(n + 1, 0);
  for (size_t i = 0; i < n; ++i) offs[i + 1] = offs[i] + b[i]->m;
  std::vector<int32_t> rows(std::max<uint64_t>(offs[n], 1) * 21);
  std::vector<uint8_t> res(sequence ? std::max<uint64_t>(offs[n], 1) : 0);
  for (size_t i = 0; i < n; ++i) {
    if (b[i]->m) memcpy(rows.data() + offs[i] * 21, b[i]->rows.data(), b[i]->rows.size() * 4);
    if (sequence && b[i]->m) memcpy(res.data() + offs[i], b[i]->residues.data(), b[i]->m);
  }
  std::vector<uint32_t> ids(n);
  int rc = st_profiles_create(ctx, rows.data(), offs.data(), static_cast<uint32_t>(n), ids.data());
  if (rc != ST_OK) return rc;
  std::unordered_map<uint32_t, uint32_t> at;  // profile id -> request
  for (size_t i = 0; i < n; ++i) at[ids[i]] = static_cast<uint32_t>(i);
  // room for 1,024 candidates per query; a batch with more runs again with the exact room
  std::vector<st_candidate> cands(std::max<size_t>(n * 1024, 65536));
  uint64_t nc = 0;
  rc = st_prefilter_queries(ctx, ids.data(), static_cast<uint32_t>(n), sequence ? res.data() : nullptr,
                            sequence ? offs.data() : nullptr, &sp, &gp, cands.data(), cands.size(), &nc, nullptr,
                            nullptr);
  if (rc == ST_OK && nc > cands.size()) {
    cands.resize(nc);
    rc = st_prefilter_queries(ctx, ids.data(), static_cast<uint32_t>(n), sequence ? res.data() : nullptr,
                              sequence ? offs.data() : nullptr, &sp, &gp, cands.data(), nc, &nc, nullptr, nullptr);
  }
  cands.resize(rc == ST_OK ? nc : 0);
  std::vector<int32_t> scores(cands.size());
  if (rc == ST_OK && !cands.empty()) {
    std::vector<st_pair> pairs(cands.size());
    for (size_t k = 0; k < cands.size(); ++k) pairs[k] = st_pair{cands[k].query, cands[k].target, 0, -1};
    rc = st_sw_score_pairs(ctx, pairs.data(), pairs.size(), gp.gap_open, gp.gap_ext, scores.data(), nullptr);
  }
  st_profiles_free(ctx, ids.data(), static_cast<uint32_t>(n));
  if (rc != ST_OK) return rc;
  for (auto& r : b) {
    r->cands.clear();
    r->scores.clear();
  }
  for (size_t k = 0; k < cands.size(); ++k) {
    auto& r = b[at[cands[k].query]];
    st_candidate c = cands[k];
    c.query = 0;
    r->cands.push_back(c);
    r->scores.push_back(scores[k]);
  }
  return ST_OK;
}

void st_search_server::run() {
  for (;;) {
    std::vector<std::shared_ptr<SearchRequest>> b;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return stop || !pending.empty(); });
      if (stop && pending.empty()) return;
      while (!pending.empty() && b.size() < max_queries) {
        b.push_back(pending.front());
        pending.pop_front();
      }
    }
    const int rc = search(b);
    const std::string err = rc == ST_OK ? std::string() : std::string(st_last_error());
    const Clock::time_point now = Clock::now();
    std::lock_guard<std::mutex> lk(mu);
    for (auto& r : b) {
      r->status = rc;
      r->error = err;
      r->t_done = now;
      r->done = true;
    }
    ++batches;
    queries += b.size();
    cv_done.notify_all();
  }
}

extern "C" st_search_server* st_search_server_create(st_ctx* ctx, const st_seed_params* seed_params,
                                                     const st_prefilter_params* params, int sequence_queries,
                                                     uint32_t max_batch_queries) {
  if (!ctx || !seed_params || !params) {
    st_internal_set_error("st_search_server_create: null argument");
    return nullptr;
  }
  auto s = std::make_unique<st_search_server>();
  s->ctx = ctx;
  s->sp = *seed_params;
  s->gp = *params;
  s->sequence = sequence_queries != 0;
  s->max_queries = max_batch_queries ? max_batch_queries : 4096;
  st_search_server* p = s.get();
  s->worker = std::thread([p] { p->run(); });
  return s.release();
}

extern "C" int st_search_server_submit(st_search_server* s, const int32_t* rows, uint32_t m, const uint8_t* residues,
                                       uint64_t* request_id) {
  if (!s || !request_id || (m && !rows) || (s->sequence && m && !residues)) {
    st_internal_set_error("st_search_server_submit: null argument");
    return ST_EINVAL;
  }
  auto r = std::make_shared<SearchRequest>();
  r->m = m;
  r->rows.assign(rows, rows + static_cast<size_t>(m) * 21);
  if (s->sequence) r->residues.assign(residues, residues + m);
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) {
    st_internal_set_error("st_search_server_submit: server is stopping");
    return ST_ESTATE;
  }
  r->id = s->next_id++;
  r->t_submit = Clock::now();
  s->live[r->id] = r;
  s->pending.push_back(r);
  *request_id = r->id;
  s->cv_work.notify_one();
  return ST_OK;
}

extern "C" int st_search_server_wait(st_search_server* s, uint64_t request_id, st_candidate* cands, int32_t* scores,
                                     uint64_t cap, uint64_t* n_out, double* latency_ms) {
  if (!s || !n_out) {
    st_internal_set_error("st_search_server_wait: null argument");
    return ST_EINVAL;
  }
  std::shared_ptr<SearchRequest> r;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->live.find(request_id);
    if (it == s->live.end()) {
      st_internal_set_error("st_search_server_wait: unknown request id");
      return ST_EINVAL;
    }
    r = it->second;
    s->cv_done.wait(lk, [&] { return r->done; });
  }
  if (r->status != ST_OK) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->live.erase(request_id);
    st_internal_set_error(r->error.c_str());
    return r->status;
  }
  *n_out = r->cands.size();
  if (cap < r->cands.size()) return ST_OK;  // call again with room for *n_out (the request stays)
  if (cands) memcpy(cands, r->cands.data(), r->cands.size() * sizeof(st_candidate));
  if (scores) memcpy(scores, r->scores.data(), r->scores.size() * 4);
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  std::lock_guard<std::mutex> lk(s->mu);
  s->live.erase(request_id);
  return ST_OK;
}

extern "C" int st_search_server_stats(st_search_server* s, uint64_t* batches, uint64_t* queries) {
  if (!s) {
    st_internal_set_error("st_search_server_stats: null server");
    return ST_EINVAL;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (batches) *batches = s->batches;
  if (queries) *queries = s->queries;
  return ST_OK;
}

extern "C" void st_search_server_destroy(st_search_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  delete s;
}
