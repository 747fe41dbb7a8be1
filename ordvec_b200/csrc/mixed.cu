// Mixed batches: many queries, each searched in its own RankQuant index (the
// same corpus at bits 1 / 2 / 4, say) for its own k, in one call.
//
// Queries are grouped by index; a group runs as one batched full search with
// the group's largest k and each query's row keeps its own first k (the top-k
// is a prefix of the top-k_max, ties by id included), padded with (-inf, -1).
//
// A group on the split-BF16 tensor-core path whose key matrix fits one chunk
// runs through a plan cached per (device, index, rows, queries, k): the plan
// owns a stream and its buffers.  Its first call runs the exact pipeline
// (which settles the candidate count kp), times the tensor-core scan at 32,
// 64 and 128 queries per tile on a slice of the index and keeps the fastest
// (the autotuner), then captures the whole pipeline -- split, scan, candidate
// select, margin test, FP64 rescoring, final select, result conversion -- as
// a CUDA graph with the fixed kp.  Later calls copy the queries in, replay the
// graph and read back the results and the margin flag; if the flag shows kp
// was too small for some query (its result would not be exact), the call
// reruns the exact pipeline and the plan is captured again with the larger kp.
#include <cmath>
#include <limits>
#include <map>
#include <mutex>
#include <tuple>

#include "ovb_host.h"

namespace ovb {

namespace {

struct Plan {
  const Index* ix = nullptr;
  uint64_t nq = 0;
  uint32_t k = 0;
  std::unique_ptr<Workspace> w;
  DevBuf dq, ds, di, dflag;
  HostBuf hflag;
  uint64_t kp = 0;
  uint32_t qpt = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t replays = 0;
  bool no_graph = false;  // capture failed once: keep to the exact pipeline
  std::mutex mu;
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  ~Plan() { drop_graph(); }
};

using PlanKey = std::tuple<int, const Index*, uint64_t, uint64_t, uint32_t>;  // device, index, rows, nq, k
std::mutex g_mu;
std::map<PlanKey, std::unique_ptr<Plan>> g_plans;

bool graphs_enabled() {
  const char* e = getenv("OVB_MIXED_GRAPH");
  return !(e && e[0] == '0');
}

float inv_norm_of(uint32_t dim, uint32_t bits) {
  const double n = (double)(1u << bits);
  return 1.0f / (float)std::sqrt((double)dim * ((n * n - 1.0) / 12.0));
}

// The autotuner: event-time the scan at 32 / 64 / 128 queries per tile over
// the first (up to) 64K rows with the plan's split queries, keep the fastest.
uint32_t autotune_tile(Plan& p) {
  Workspace& w = *p.w;
  const Index& ix = *p.ix;
  const uint64_t rows = std::min<uint64_t>(ix.n, 65536);
  uint32_t* keys = (uint32_t*)w.keys.ensure(p.nq * rows * 4);  // tuning scans write rows x nq keys
  const float inv_norm = inv_norm_of(ix.dim, ix.bits);
  cudaEvent_t e0, e1;
  OVB_CUDA(cudaEventCreate(&e0));
  OVB_CUDA(cudaEventCreate(&e1));
  uint32_t best = 128;
  float best_ms = std::numeric_limits<float>::infinity();
  for (uint32_t qpt : {32u, 64u, 128u}) {
    if (qpt > 32 && (uint64_t)qpt / 2 >= p.nq) break;  // larger tiles than the batch change nothing
    launch_rank_scan_tc(ix.codes.as<uint8_t>(), rows, ix.dim, ix.bits, w.q_split.p, p.nq, inv_norm, 1, keys, rows,
                        qpt, w.tc_err_word(w.stream), w.stream);
    OVB_CUDA(cudaEventRecord(e0, w.stream));
    for (int r = 0; r < 2; r++)
      launch_rank_scan_tc(ix.codes.as<uint8_t>(), rows, ix.dim, ix.bits, w.q_split.p, p.nq, inv_norm, 1, keys, rows,
                          qpt, w.tc_err_word(w.stream), w.stream);
    OVB_CUDA(cudaEventRecord(e1, w.stream));
    OVB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    OVB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best_ms) {
      best_ms = ms;
      best = qpt;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  check_tc_errors(w);
  return best;
}

void capture(Plan& p) {
  Workspace& w = *p.w;
  cudaStream_t st = w.stream;
  uint32_t* flag = (uint32_t*)p.dflag.ensure(4);
  OVB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  try {
    OVB_CUDA(cudaMemsetAsync(flag, 0, 4, st));
    const uint32_t ke = engine_rankquant_split_fixed(*p.ix, p.dq.as<float>(), p.nq, p.k, p.kp, p.qpt, flag, w, st);
    launch_keys_to_results(w.out_keys.as<uint32_t>(), w.out_ids.as<uint32_t>(), p.nq * ke, 0, 0, p.ds.as<float>(),
                           p.di.as<int64_t>(), st);
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(st, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  OVB_CUDA(cudaStreamEndCapture(st, &p.graph));
  OVB_CUDA(cudaGraphInstantiate(&p.exec, p.graph, 0));
}

// Runs one group through its plan in two phases, so the groups of a mixed
// batch overlap on the device: plan_enqueue copies the queries in and, once a
// graph exists, replays it and queues the copies of the margin flag and the
// results (host in, host out, nothing waited for); plan_finish waits for the
// plan's stream and, on the first call or when the flag shows kp was too small
// for some query, runs the exact pipeline and (re)captures the graph.
bool plan_enqueue(Plan& p, const float* h_q, float* h_s, int64_t* h_i) {
  Workspace& w = *p.w;
  cudaStream_t st = w.stream;
  const Index& ix = *p.ix;
  const uint32_t ke = (uint32_t)std::min<uint64_t>(p.k, ix.n);
  float* dq = (float*)p.dq.ensure(p.nq * ix.dim * 4);
  float* ds = (float*)p.ds.ensure(p.nq * ke * 4);
  int64_t* di = (int64_t*)p.di.ensure(p.nq * ke * 8);
  uint32_t* hflag = (uint32_t*)p.hflag.ensure(4);
  OVB_CUDA(cudaMemcpyAsync(dq, h_q, p.nq * ix.dim * 4, cudaMemcpyHostToDevice, st));
  if (!p.exec) return false;
  OVB_CUDA(cudaGraphLaunch(p.exec, st));
  OVB_CUDA(cudaMemcpyAsync(hflag, p.dflag.p, 4, cudaMemcpyDeviceToHost, st));
  OVB_CUDA(cudaMemcpyAsync(h_s, ds, p.nq * ke * 4, cudaMemcpyDeviceToHost, st));
  OVB_CUDA(cudaMemcpyAsync(h_i, di, p.nq * ke * 8, cudaMemcpyDeviceToHost, st));
  return true;
}

void plan_finish(Plan& p, bool enqueued, float* h_s, int64_t* h_i) {
  Workspace& w = *p.w;
  cudaStream_t st = w.stream;
  const Index& ix = *p.ix;
  const uint32_t ke = (uint32_t)std::min<uint64_t>(p.k, ix.n);
  OVB_CUDA(cudaStreamSynchronize(st));
  bool done = false;
  if (enqueued) {
    check_tc_errors(w);
    p.replays++;
    done = *(uint32_t*)p.hflag.p == 0;
  }
  if (done) return;
  // first call, or kp was too small for some query: the exact pipeline
  float* dq = p.dq.as<float>();
  float* ds = p.ds.as<float>();
  int64_t* di = p.di.as<int64_t>();
  engine_rankquant_full_split(ix, dq, p.nq, p.k, true, w, st, p.qpt);
  launch_keys_to_results(w.out_keys.as<uint32_t>(), w.out_ids.as<uint32_t>(), p.nq * ke, 0, 0, ds, di, st);
  OVB_CUDA(cudaStreamSynchronize(st));
  check_tc_errors(w);
  const uint64_t kp = std::max<uint64_t>(w.split_kp, ke);
  if (!p.no_graph && (!p.exec || kp > p.kp)) {
    p.drop_graph();
    p.kp = kp;
    if (!p.qpt) p.qpt = autotune_tile(p);
    try {
      capture(p);
    } catch (const CudaError&) {
      p.drop_graph();
      p.no_graph = true;
      cudaGetLastError();
    }
  }
  OVB_CUDA(cudaMemcpyAsync(h_s, ds, p.nq * ke * 4, cudaMemcpyDeviceToHost, st));
  OVB_CUDA(cudaMemcpyAsync(h_i, di, p.nq * ke * 8, cudaMemcpyDeviceToHost, st));
  OVB_CUDA(cudaStreamSynchronize(st));
}

Plan& plan_for(const Index& ix, uint64_t nq, uint32_t k) {
  int dev = 0;
  OVB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_mu);
  auto& slot = g_plans[PlanKey{dev, &ix, ix.n, nq, k}];
  if (!slot) {
    slot.reset(new Plan());
    slot->ix = &ix;
    slot->nq = nq;
    slot->k = k;
    slot->w.reset(new Workspace());
  }
  return *slot;
}

}  // namespace

void mixed_forget_index(const Index* ix) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto it = g_plans.begin(); it != g_plans.end();) {
    if (std::get<1>(it->first) == ix)
      it = g_plans.erase(it);
    else
      ++it;
  }
}

bool mixed_plan_info(const Index& ix, uint64_t nq, uint64_t k, uint32_t* qpt, uint64_t* kp, uint64_t* replays) {
  int dev = 0;
  OVB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_plans.find(PlanKey{dev, &ix, ix.n, nq, (uint32_t)k});
  if (it == g_plans.end()) return false;
  *qpt = it->second->qpt;
  *kp = it->second->kp;
  *replays = it->second->replays;
  return true;
}

// Whether a group of nq queries of index ix with top-k runs through a plan.
bool group_uses_plan(const Index& ix, uint64_t nq, uint64_t k) {
  return graphs_enabled() && rank_tc_eligible(ix.dim, ix.bits) && split_fixed_fits(ix, nq, k);
}

// One group without a plan: nq queries of one index with k; host in, host out (nq x ke).
uint32_t mixed_group_direct(const Index& ix, const float* h_q, uint64_t nq, uint64_t k, float* h_s, int64_t* h_i) {
  const uint32_t ke = (uint32_t)std::min<uint64_t>(k, ix.n);
  if (!ke || !nq) return ke;
  Workspace& w = workspace();
  float* dq = (float*)w.q_raw.ensure(nq * ix.dim * 4);
  OVB_CUDA(cudaMemcpyAsync(dq, h_q, nq * ix.dim * 4, cudaMemcpyHostToDevice, w.stream));
  const uint32_t got = engine_rankquant_full(ix, dq, nq, ke, w, w.stream);
  float* ds = (float*)w.scores.ensure(nq * got * 4);
  int64_t* di = (int64_t*)w.ids.ensure(nq * got * 8);
  launch_keys_to_results(w.out_keys.as<uint32_t>(), w.out_ids.as<uint32_t>(), nq * got, 0, 0, ds, di, w.stream);
  OVB_CUDA(cudaMemcpyAsync(h_s, ds, nq * got * 4, cudaMemcpyDeviceToHost, w.stream));
  OVB_CUDA(cudaMemcpyAsync(h_i, di, nq * got * 8, cudaMemcpyDeviceToHost, w.stream));
  OVB_CUDA(cudaStreamSynchronize(w.stream));
  check_tc_errors(w);
  return got;
}

}  // namespace ovb

using namespace ovb;

ordvec_status_t ovb_rankquant_search_mixed(const ordvec_index_t* const* indices, uint32_t n_indices,
                                           const uint32_t* index_of_query, const uint32_t* k_of_query,
                                           const float* queries, uint64_t nq, uint64_t k_max, float* scores,
                                           int64_t* ids) {
  return api_boundary([&] {
    if (!nq) return;
    if (!indices || !index_of_query || !k_of_query || !queries) fail(ORDVEC_STATUS_NULL_POINTER, "input pointer is NULL");
    if (!n_indices) fail(ORDVEC_STATUS_BAD_ARGUMENT, "n_indices must be positive");
    std::vector<const Index*> ix(n_indices);
    for (uint32_t j = 0; j < n_indices; j++) {
      ix[j] = &as_index(indices[j]);
      if (ix[j]->kind != ORDVEC_INDEX_KIND_RANK_QUANT)
        fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "mixed search: every index must be RankQuant");
      if (ix[j]->dim != ix[0]->dim) fail(ORDVEC_STATUS_DIM_MISMATCH, "mixed search: indices differ in dim");
    }
    const uint32_t dim = ix[0]->dim;
    std::vector<std::vector<uint64_t>> groups(n_indices);
    for (uint64_t i = 0; i < nq; i++) {
      if (index_of_query[i] >= n_indices) fail(ORDVEC_STATUS_BAD_ARGUMENT, "index_of_query out of range");
      if (k_of_query[i] > k_max) fail(ORDVEC_STATUS_BAD_ARGUMENT, "k_of_query exceeds k_max");
      groups[index_of_query[i]].push_back(i);
    }
    for (uint64_t v = 0; v < nq * dim; v++)
      if (!std::isfinite(queries[v])) fail(ORDVEC_STATUS_NONFINITE_QUERY, "query contains NaN or infinity");
    if (k_max && (!scores || !ids)) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    for (uint64_t v = 0; v < nq * k_max; v++) {
      scores[v] = -std::numeric_limits<float>::infinity();
      ids[v] = -1;
    }
    // pinned staging per group: the groups' copies and replays are in flight together
    thread_local std::vector<std::unique_ptr<HostBuf>> sq, ss, si;
    while (sq.size() < n_indices) {
      sq.emplace_back(new HostBuf());
      ss.emplace_back(new HostBuf());
      si.emplace_back(new HostBuf());
    }
    auto stage_q = [&](uint32_t j) -> HostBuf& { return *sq[j]; };
    auto stage_s = [&](uint32_t j) -> HostBuf& { return *ss[j]; };
    auto stage_i = [&](uint32_t j) -> HostBuf& { return *si[j]; };
    std::vector<uint64_t> kg(n_indices, 0), keg(n_indices, 0);
    std::vector<Plan*> plan(n_indices, nullptr);
    std::vector<std::unique_lock<std::mutex>> locks;
    std::vector<char> enqueued(n_indices, 0);
    // phase 1: stage every group; groups with a plan replay its graph (no wait)
    for (uint32_t j = 0; j < n_indices; j++) {
      const auto& g = groups[j];
      if (g.empty()) continue;
      for (uint64_t i : g) kg[j] = std::max<uint64_t>(kg[j], k_of_query[i]);
      const uint64_t nqg = g.size();
      keg[j] = std::min<uint64_t>(kg[j], ix[j]->n);
      float* hq = (float*)stage_q(j).ensure(nqg * dim * 4);
      stage_s(j).ensure(std::max<uint64_t>(nqg * keg[j], 1) * 4);
      stage_i(j).ensure(std::max<uint64_t>(nqg * keg[j], 1) * 8);
      for (uint64_t r = 0; r < nqg; r++) std::copy(queries + g[r] * dim, queries + (g[r] + 1) * dim, hq + r * dim);
      if (keg[j] && group_uses_plan(*ix[j], nqg, kg[j])) {
        plan[j] = &plan_for(*ix[j], nqg, (uint32_t)keg[j]);
        locks.emplace_back(plan[j]->mu);  // plans of one call are distinct; taken in group order
        enqueued[j] = plan_enqueue(*plan[j], hq, (float*)stage_s(j).p, (int64_t*)stage_i(j).p);
      }
    }
    // phase 2: finish every group and scatter its rows (each row keeps its own k)
    for (uint32_t j = 0; j < n_indices; j++) {
      const auto& g = groups[j];
      if (g.empty() || !keg[j]) continue;
      const uint64_t nqg = g.size();
      float* hs = (float*)stage_s(j).p;
      int64_t* hi = (int64_t*)stage_i(j).p;
      uint64_t got;
      if (plan[j]) {
        plan_finish(*plan[j], enqueued[j] != 0, hs, hi);
        got = keg[j];
      } else {
        got = mixed_group_direct(*ix[j], (const float*)stage_q(j).p, nqg, kg[j], hs, hi);
      }
      for (uint64_t r = 0; r < nqg; r++) {
        const uint64_t i = g[r];
        const uint64_t keep = std::min<uint64_t>(k_of_query[i], got);
        std::copy(hs + r * got, hs + r * got + keep, scores + i * k_max);
        std::copy(hi + r * got, hi + r * got + keep, ids + i * k_max);
      }
    }
  });
}

ordvec_status_t ovb_mixed_plan_info(const ordvec_index_t* rq, uint64_t nq, uint64_t k, uint32_t* q_per_tile,
                                    uint64_t* candidates, uint64_t* replays) {
  return api_boundary([&] {
    const Index& ix = as_index(rq);
    if (!q_per_tile || !candidates || !replays) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    if (!mixed_plan_info(ix, nq, std::min<uint64_t>(k, ix.n), q_per_tile, candidates, replays))
      fail(ORDVEC_STATUS_BAD_ARGUMENT, "no plan for this index, batch size and k");
  });
}
