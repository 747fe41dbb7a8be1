// Serving loop: a request queue over device-resident indices, answered by
// worker threads that each own a CUDA stream and a workspace.
//
// Continuous batching: a worker that becomes free takes the oldest pending
// request and every later pending request of the same route, whatever their
// k and m, up to max_batch queries, so requests that arrived while other
// batches ran join the next batch.  A batch runs at its largest k; when its
// requests' candidate counts differ (m, or the default policy's count for
// their k) stage 1 selects each query's ordered top-m_max and each query is
// reranked over its own top-m prefix (engine_two_stage_ragged).  A request
// then takes the first min(k, m) entries of its rows: the exact top-k of a
// strict (score, id) order is a prefix of the top-k_max.  Admission: a batch
// starts only when the device bytes of all batches in flight stay within the
// HBM budget (a batch larger than the budget runs alone).  Batches of
// different workers overlap on the device.  Each query's result does not
// depend on its batch-mates (every kernel scores queries independently;
// stage-1 candidate sets and the rerank are exact per query), so a request
// gets the same answer alone and in the mix.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "ovb_host.h"

struct ovb_server {};  // opaque handle type of the C ABI

namespace ovb {

namespace {

using Clock = std::chrono::steady_clock;

struct Route {
  const Index* rq;
  const Index* s1;  // null: full RankQuant search
};

struct Request {
  uint64_t ticket = 0;
  uint32_t route = 0;
  uint64_t nq = 0, k = 0, m = 0;
  std::vector<float> q;
  Clock::time_point submitted;
  bool done = false;
  ordvec_status_t status = ORDVEC_STATUS_OK;
  std::string msg;
  uint64_t k_out = 0;
  std::vector<float> scores;
  std::vector<int64_t> ids;
  double latency_ms = 0.0;
};
using ReqPtr = std::shared_ptr<Request>;

constexpr uint64_t kServerMagic = 0x5245565245534256ull;

struct Server : ovb_server {
  uint64_t magic = kServerMagic;
  int device = 0;
  uint32_t workers = 2, max_batch = 1024;
  uint64_t budget = 4ull << 30;
  std::vector<Route> routes;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_budget;
  std::deque<ReqPtr> pending;
  std::unordered_map<uint64_t, ReqPtr> tickets;
  uint64_t next_ticket = 1;
  bool stopping = false;
  uint64_t inflight = 0, peak_inflight = 0;
  uint32_t running = 0, max_running = 0;
  uint64_t n_req = 0, n_q = 0, n_batches = 0, warm_workers = 0;
  std::vector<double> latencies;
  std::vector<std::thread> threads;
};

Server& as_server(ovb_server_t* s) {
  if (!s) fail(ORDVEC_STATUS_NULL_POINTER, "server pointer is NULL");
  Server* p = static_cast<Server*>(s);
  if (p->magic != kServerMagic) fail(ORDVEC_STATUS_BAD_ARGUMENT, "not a live server handle");
  return *p;
}

// Device bytes a batch needs: query copies, the intermediates of its stage 1
// (the sampled filter's rows, or a key matrix the engine caps at its 2 GiB
// budget) or of its full scan, candidate and result rows.
uint64_t batch_bytes(const Route& r, uint64_t nq, uint64_t k, uint64_t m) {
  const uint64_t n = r.rq->n, dim = r.rq->dim;
  const uint64_t me = r.s1 ? (m ? std::min<uint64_t>(m, n) : default_candidate_count(k, n)) : 0;
  const uint64_t keys = r.s1 ? engine_stage1_bytes(*r.s1, nq, me) : std::min<uint64_t>(nq * n * 4, 2ull << 30);
  return keys + nq * (12 * dim + 24 * me + 24 * k + 8192);
}

// Candidate count a two-stage request resolves to: its m, or the default
// policy's count for its k (src/quant.rs:234-262), clamped to n.
uint64_t resolved_m(const Route& r, const Request& q) {
  const uint64_t n = r.rq->n;
  return q.m ? std::min<uint64_t>(q.m, n) : default_candidate_count(q.k, n);
}

void run_batch(Server& S, const Route& rt, std::vector<ReqPtr>& batch, uint64_t nq, HostBuf& hq, HostBuf& hs,
               HostBuf& hi, DevBuf& dq, DevBuf& ds, DevBuf& di) {
  Workspace& w = workspace();
  const Index& r = *rt.rq;
  const uint64_t dim = r.dim;
  uint64_t k = 0;
  bool uniform = true;
  for (auto& q : batch) {
    k = std::max(k, q->k);
    uniform = uniform && resolved_m(rt, *q) == resolved_m(rt, *batch[0]);
  }
  float* hqp = (float*)hq.ensure(nq * dim * 4);
  uint64_t off = 0;
  for (auto& q : batch) {
    std::copy(q->q.begin(), q->q.end(), hqp + off * dim);
    off += q->nq;
  }
  float* d_q = (float*)dq.ensure(nq * dim * 4);
  OVB_CUDA(cudaMemcpyAsync(d_q, hqp, nq * dim * 4, cudaMemcpyHostToDevice, w.stream));
  uint32_t ke;
  if (!rt.s1) {
    ke = engine_rankquant_full(r, d_q, nq, k, w, w.stream);
  } else if (uniform) {
    ke = engine_two_stage(r, *rt.s1, d_q, nq, resolved_m(rt, *batch[0]), k, w, w.stream);
  } else {
    std::vector<uint64_t> m_of;
    m_of.reserve(nq);
    for (auto& q : batch) m_of.insert(m_of.end(), q->nq, resolved_m(rt, *q));
    ke = engine_two_stage_ragged(r, *rt.s1, d_q, nq, m_of.data(), k, w, w.stream);
  }
  float* hsp = nullptr;
  int64_t* hip = nullptr;
  if (ke) {
    float* dsp = (float*)ds.ensure(nq * ke * 4);
    int64_t* dip = (int64_t*)di.ensure(nq * ke * 8);
    launch_keys_to_results(w.out_keys.as<uint32_t>(), w.out_ids.as<uint32_t>(), nq * ke, 0, 0, dsp, dip, w.stream);
    hsp = (float*)hs.ensure(nq * ke * 4);
    hip = (int64_t*)hi.ensure(nq * ke * 8);
    OVB_CUDA(cudaMemcpyAsync(hsp, dsp, nq * ke * 4, cudaMemcpyDeviceToHost, w.stream));
    OVB_CUDA(cudaMemcpyAsync(hip, dip, nq * ke * 8, cudaMemcpyDeviceToHost, w.stream));
  }
  OVB_CUDA(cudaStreamSynchronize(w.stream));
  check_tc_errors(w);
  off = 0;
  for (auto& q : batch) {
    // this request's own width: min(k, its candidate count), a prefix of each row
    uint64_t kq = std::min<uint64_t>(q->k, ke);
    if (rt.s1) kq = std::min<uint64_t>(kq, resolved_m(rt, *q));
    q->k_out = kq;
    q->scores.resize(q->nq * kq);
    q->ids.resize(q->nq * kq);
    for (uint64_t i = 0; i < q->nq && kq; i++) {
      std::copy(hsp + (off + i) * ke, hsp + (off + i) * ke + kq, q->scores.begin() + i * kq);
      std::copy(hip + (off + i) * ke, hip + (off + i) * ke + kq, q->ids.begin() + i * kq);
    }
    off += q->nq;
  }
}

// Grow this worker's device and pinned buffers to a route's largest batch
// before it serves requests: buffers only grow, and a growth frees the old
// allocation, which waits for the whole device and would stall the other
// workers' batches mid-stream.  Both stage-1 forms are exercised (the CUDA-core
// scan with its key rows below 8 or 32 queries, and tensor-core batches).
// Two-stage routes also run a ragged batch (requests of different candidate
// counts: one query at k = 10, the rest at k = 100, the default policy's 320
// and 3,200 candidates), whose CSR offsets, compacted candidate rows and keys
// the uniform batches never size.  Requests beyond k = 100 (or explicit m
// above 3,200) may still grow buffers on first use.
void warm_route(Server& S, const Route& rt, HostBuf& hq, HostBuf& hs, HostBuf& hi, DevBuf& dq, DevBuf& ds,
                DevBuf& di) {
  const uint32_t dim = rt.rq->dim;
  auto make = [&](uint64_t nq, uint64_t k) {
    auto r = std::make_shared<Request>();
    r->nq = nq;
    r->k = k;
    r->m = 0;
    r->q.resize(nq * dim);
    uint64_t x = 0x9E3779B97F4A7C15ull ^ nq;
    for (float& v : r->q) {  // deterministic, finite, non-degenerate
      x ^= x << 13;
      x ^= x >> 7;
      x ^= x << 17;
      v = (float)((int64_t)(x >> 40) - (1 << 23)) * (1.0f / (1 << 23));
    }
    return r;
  };
  for (uint64_t nq : {(uint64_t)7, (uint64_t)31, (uint64_t)S.max_batch}) {
    if (nq > S.max_batch) continue;
    std::vector<ReqPtr> batch(1, make(nq, 100));
    run_batch(S, rt, batch, nq, hq, hs, hi, dq, ds, di);
    if (rt.s1 && nq >= 2) {
      std::vector<ReqPtr> ragged{make(1, 10), make(nq - 1, 100)};
      run_batch(S, rt, ragged, nq, hq, hs, hi, dq, ds, di);
    }
  }
}

void worker_main(Server* S) {
  cudaSetDevice(S->device);
  HostBuf hq, hs, hi;
  DevBuf dq, ds, di;
  size_t warmed = 0;  // routes this worker has pre-sized its buffers for
  for (;;) {
    std::vector<ReqPtr> batch;
    uint64_t nq = 0, bytes = 0;
    Route rt{};
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] { return S->stopping || !S->pending.empty() || warmed < S->routes.size(); });
      if (warmed < S->routes.size()) {
        const Route w = S->routes[warmed++];
        lk.unlock();
        api_boundary([&] { warm_route(*S, w, hq, hs, hi, dq, ds, di); });
        lk.lock();
        if (warmed == S->routes.size()) S->warm_workers++;
        continue;
      }
      if (S->pending.empty()) return;  // stopping and drained
      // the oldest request, then every later one of the same route
      const ReqPtr head = S->pending.front();
      uint64_t k_max = 0, m_max = 0;
      for (auto it = S->pending.begin(); it != S->pending.end();) {
        const ReqPtr& q = *it;
        const bool same = q->route == head->route;
        if (same && (batch.empty() || nq + q->nq <= S->max_batch)) {
          k_max = std::max(k_max, q->k);
          m_max = std::max(m_max, q->m ? q->m : default_candidate_count(q->k, S->routes[q->route].rq->n));
          nq += q->nq;
          batch.push_back(q);
          it = S->pending.erase(it);
        } else {
          ++it;
        }
      }
      rt = S->routes[head->route];
      bytes = batch_bytes(rt, nq, k_max, m_max);
      S->cv_budget.wait(lk, [&] { return S->inflight == 0 || S->inflight + bytes <= S->budget; });
      S->inflight += bytes;
      S->peak_inflight = std::max(S->peak_inflight, S->inflight);
      S->running++;
      S->max_running = std::max(S->max_running, S->running);
      if (!S->pending.empty()) S->cv_work.notify_one();  // another worker may take the rest
    }
    ordvec_status_t st = api_boundary([&] { run_batch(*S, rt, batch, nq, hq, hs, hi, dq, ds, di); });
    const char* err = st == ORDVEC_STATUS_OK ? nullptr : ordvec_last_error();
    const Clock::time_point now = Clock::now();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->inflight -= bytes;
      S->running--;
      S->n_batches++;
      for (auto& q : batch) {
        q->status = st;
        if (err) q->msg = err;
        q->latency_ms = std::chrono::duration<double, std::milli>(now - q->submitted).count();
        q->done = true;
        if (st == ORDVEC_STATUS_OK) {
          S->n_req++;
          S->n_q += q->nq;
          S->latencies.push_back(q->latency_ms);
        }
      }
    }
    S->cv_done.notify_all();
    S->cv_budget.notify_all();
  }
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = p * (double)(v.size() - 1);
  const size_t lo = (size_t)std::floor(pos), hi = std::min(lo + 1, v.size() - 1);
  return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace
}  // namespace ovb

using namespace ovb;

ordvec_status_t ovb_server_new(const ovb_server_config_t* config, ovb_server_t** out) {
  return api_boundary([&] {
    if (!out) fail(ORDVEC_STATUS_NULL_POINTER, "out pointer is NULL");
    *out = nullptr;
    if (!config) fail(ORDVEC_STATUS_NULL_POINTER, "config pointer is NULL");
    if (config->struct_size != sizeof(ovb_server_config_t))
      fail(ORDVEC_STATUS_BAD_STRUCT_SIZE, "ovb_server_config_t.struct_size must be exactly " +
                                              std::to_string(sizeof(ovb_server_config_t)));
    for (uint64_t r : config->reserved)
      if (r) fail(ORDVEC_STATUS_BAD_ARGUMENT, "ovb_server_config_t.reserved must be zero");
    if (config->workers > 64) fail(ORDVEC_STATUS_BAD_ARGUMENT, "workers must be at most 64");
    ensure_device();
    std::unique_ptr<Server> s(new Server());
    OVB_CUDA(cudaGetDevice(&s->device));
    if (config->workers) s->workers = config->workers;
    if (config->max_batch) s->max_batch = config->max_batch;
    if (config->hbm_budget_bytes) s->budget = config->hbm_budget_bytes;
    Server* raw = s.get();
    for (uint32_t i = 0; i < s->workers; i++) s->threads.emplace_back(worker_main, raw);
    *out = s.release();
  });
}

ordvec_status_t ovb_server_add_route(ovb_server_t* server, const ordvec_index_t* rq, const ordvec_index_t* stage1,
                                     uint32_t* route_out) {
  return api_boundary([&] {
    Server& S = as_server(server);
    if (!route_out) fail(ORDVEC_STATUS_NULL_POINTER, "route_out pointer is NULL");
    const Index& r = as_index(rq);
    if (r.kind != ORDVEC_INDEX_KIND_RANK_QUANT) fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "route: rq must be RankQuant");
    const Index* s1 = nullptr;
    if (stage1) {
      s1 = &as_index(stage1);
      if (s1->kind == ORDVEC_INDEX_KIND_RANK_QUANT)
        fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "route: stage 1 must be a candidate-generating index");
      if (s1->dim != r.dim) fail(ORDVEC_STATUS_DIM_MISMATCH, "route: stage-1 dim must match RankQuant dim");
      if (s1->n != r.n) fail(ORDVEC_STATUS_BAD_ARGUMENT, "route: stage-1 len must match RankQuant len");
    }
    std::lock_guard<std::mutex> lk(S.mu);
    S.routes.push_back(Route{&r, s1});
    *route_out = (uint32_t)(S.routes.size() - 1);
    S.warm_workers = 0;      // every worker now has a route to pre-size for
    S.cv_work.notify_all();
  });
}

ordvec_status_t ovb_server_submit(ovb_server_t* server, uint32_t route, const float* queries, uint64_t nq,
                                  uint64_t k, uint64_t m, uint64_t* ticket_out) {
  return api_boundary([&] {
    Server& S = as_server(server);
    if (!ticket_out) fail(ORDVEC_STATUS_NULL_POINTER, "ticket_out pointer is NULL");
    if (nq && !queries) fail(ORDVEC_STATUS_NULL_POINTER, "queries pointer is NULL");
    uint32_t dim;
    {
      std::lock_guard<std::mutex> lk(S.mu);
      if (route >= S.routes.size()) fail(ORDVEC_STATUS_BAD_ARGUMENT, "unknown route");
      dim = S.routes[route].rq->dim;
    }
    ReqPtr q = std::make_shared<Request>();
    q->route = route;
    q->nq = nq;
    q->k = k;
    q->m = m;
    q->q.assign(queries, queries + nq * dim);
    for (float v : q->q)
      if (!std::isfinite(v)) fail(ORDVEC_STATUS_NONFINITE_QUERY, "query contains NaN or infinity");
    q->submitted = Clock::now();
    std::lock_guard<std::mutex> lk(S.mu);
    q->ticket = S.next_ticket++;
    S.tickets[q->ticket] = q;
    if (!nq || !k) {
      q->done = true;  // nothing to compute: an empty result
    } else {
      S.pending.push_back(q);
      S.cv_work.notify_one();
    }
    *ticket_out = q->ticket;
  });
}

ordvec_status_t ovb_server_wait(ovb_server_t* server, uint64_t ticket, float* scores, int64_t* ids,
                                uint64_t capacity, uint64_t* k_out, double* latency_ms) {
  return api_boundary([&] {
    Server& S = as_server(server);
    std::unique_lock<std::mutex> lk(S.mu);
    auto it = S.tickets.find(ticket);
    if (it == S.tickets.end()) fail(ORDVEC_STATUS_BAD_ARGUMENT, "unknown or already collected ticket");
    ReqPtr q = it->second;
    S.cv_done.wait(lk, [&] { return q->done; });
    if (q->status != ORDVEC_STATUS_OK) {
      S.tickets.erase(it);
      fail(q->status, q->msg);
    }
    const uint64_t count = q->nq * q->k_out;
    if (count && (!scores || !ids)) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    if (count > capacity) fail(ORDVEC_STATUS_BUFFER_TOO_SMALL, "result needs " + std::to_string(count) + " entries");
    std::copy(q->scores.begin(), q->scores.end(), scores);
    std::copy(q->ids.begin(), q->ids.end(), ids);
    if (k_out) *k_out = q->k_out;
    if (latency_ms) *latency_ms = q->latency_ms;
    S.tickets.erase(it);
  });
}

ordvec_status_t ovb_server_stats(ovb_server_t* server, ovb_server_stats_t* out) {
  return api_boundary([&] {
    Server& S = as_server(server);
    if (!out) fail(ORDVEC_STATUS_NULL_POINTER, "out pointer is NULL");
    if (out->struct_size != sizeof(ovb_server_stats_t))
      fail(ORDVEC_STATUS_BAD_STRUCT_SIZE,
           "ovb_server_stats_t.struct_size must be exactly " + std::to_string(sizeof(ovb_server_stats_t)));
    std::lock_guard<std::mutex> lk(S.mu);
    out->requests = S.n_req;
    out->queries = S.n_q;
    out->batches = S.n_batches;
    out->peak_inflight_bytes = S.peak_inflight;
    out->max_concurrent_batches = S.max_running;
    out->warm_workers = S.warm_workers;
    out->p50_ms = percentile(S.latencies, 0.50);
    out->p99_ms = percentile(S.latencies, 0.99);
    double sum = 0.0;
    for (double v : S.latencies) sum += v;
    out->mean_ms = S.latencies.empty() ? 0.0 : sum / (double)S.latencies.size();
  });
}

void ovb_server_free(ovb_server_t* server) {
  if (!server) return;
  Server* S = static_cast<Server*>(server);
  if (S->magic != kServerMagic) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stopping = true;
  }
  S->cv_work.notify_all();
  for (auto& t : S->threads) t.join();
  S->magic = 0;
  delete S;
}
