// Internal host-side types of libordvec_b200: index handles, device buffers,
// per-thread workspaces and the status-carrying exception used at the C ABI.
#pragma once
#include <stdint.h>

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "../../include/ordvec_b200.h"
#include "ovb_common.cuh"
#include "ovb_kernels.h"

namespace ovb {

struct ApiError {
  ordvec_status_t status;
  std::string msg;
};
[[noreturn]] inline void fail(ordvec_status_t s, std::string m) { throw ApiError{s, std::move(m)}; }

// Grow-only device allocation.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  void* ensure(size_t bytes) {
    if (bytes > cap) {
      if (p) cudaFree(p);
      p = nullptr;
      cap = 0;
      OVB_CUDA(cudaMalloc(&p, bytes));
      cap = bytes;
    }
    return p;
  }
  template <class T>
  T* as() const {
    return (T*)p;
  }
};

// Grow-only pinned host allocation.
struct HostBuf {
  void* p = nullptr;
  size_t cap = 0;
  HostBuf() = default;
  HostBuf(const HostBuf&) = delete;
  HostBuf& operator=(const HostBuf&) = delete;
  ~HostBuf() {
    if (p) cudaFreeHost(p);
  }
  void* ensure(size_t bytes) {
    if (bytes > cap) {
      if (p) cudaFreeHost(p);
      p = nullptr;
      cap = 0;
      OVB_CUDA(cudaMallocHost(&p, bytes));
      cap = bytes;
    }
    return p;
  }
};

constexpr uint64_t kIndexMagic = 0x5849303032424F56ull;
constexpr uint64_t kMaxVectors = 64ull * 1024 * 1024;  // src/rank_io.rs:136
constexpr uint32_t kMaxDim = 65535;                     // src/rank_io.rs:119
constexpr uint64_t kMaxSignDim = 1ull << 24;            // src/rank_io.rs:126
constexpr uint32_t kMaxDeviceRankDim = 16384;           // device rank transform limit

struct Index {
  uint64_t magic = kIndexMagic;
  uint32_t kind = 0, dim = 0, bits = 0, n_top = 0, pairs_pad = 0;
  uint64_t n = 0;
  uint64_t file_size = 0;
  int device = 0;
  DevBuf codes;

  uint32_t qpv() const { return dim / 64; }
  uint32_t nb() const { return 1u << bits; }
  uint64_t bpv() const { return (uint64_t)dim * bits / 8; }
  // bytes_per_vec as the reference reports it
  uint64_t ref_bytes_per_vec() const;
  // device bytes holding n rows
  uint64_t device_bytes(uint64_t rows) const;
};

// Per-thread device scratch and stream.
struct Workspace {
  int device = 0;
  cudaStream_t stream = nullptr;
  DevBuf q_raw, q_unit, qbits, lut, bias, invq, keys, sel_keys, sel_ids, off, keys2, out_keys,
      out_ids, scores, ids, scratch, stage, weights, flag;
  // FastScan threshold filter: sample key matrix, per-query thresholds,
  // kept (key, id) rows, their counts and the failure flag
  DevBuf smp_keys, thr_keys, thr_ids, f_keys, f_ids, f_cnt, f_flag;
  // split-BF16 rank scan: [hi; lo] query rows and |q|_1
  DevBuf q_split, q_l1;
  // bitmap filter on FP4 tensor cores: the query bits as e2m1 nibbles
  DevBuf q_nib;
  // split-BF16 rerank: top-kp split keys / ids per query, their FP64 keys, the margin flag
  DevBuf rr_keys, rr_ids, rr_keys2, rr_flag;
  HostBuf rr_flag_host;
  // how engine_two_stage reranks (OVB_RERANK_* of ordvec_b200.h; 0 = auto)
  uint32_t rerank_mode = 0;
  // per-query candidate counts of a ragged two-stage batch: CSR offsets and rows
  HostBuf off_host;
  DevBuf csr_ids;
  uint64_t split_kp = 0;  // largest candidate count the last exact split search settled on
  bool cand_unordered = false;  // set while a two-stage search selects its stage-1 set
  HostBuf pinned, f_flag_host;
  // error word of the tensor-core kernels (zeroed once; checked by host APIs)
  DevBuf tc_err;
  bool tc_used = false;
  uint32_t* tc_err_word(cudaStream_t st) {
    if (!tc_err.p) {
      tc_err.ensure(4);
      OVB_CUDA(cudaMemsetAsync(tc_err.p, 0, 4, st));
    }
    tc_used = true;
    return tc_err.as<uint32_t>();
  }
  // stage markers for ovb_two_stage_profile (recorded only while prof is set):
  // 0 start, 1 query prep, 6 candidate threshold, 2 scan, 3 select, 4 rerank,
  // 5 final select
  cudaEvent_t prof_ev[7] = {};
  bool prof = false;
  void mark(cudaStream_t st, int i) {
    if (prof) OVB_CUDA(cudaEventRecord(prof_ev[i], st));
  }
  Workspace();
  ~Workspace();
};

Workspace& workspace();
const Index& as_index(const ordvec_index_t* h);
Index& as_index_mut(ordvec_index_t* h);
void ensure_device();

// pipelines on device pointers (engine.cpp); return the effective k
uint32_t engine_rankquant_full(const Index& rq, const float* d_q, uint64_t nq, uint64_t k,
                               Workspace& w, cudaStream_t st);
// Full search scored by the split-BF16 tensor-core scan; exact = true rescores
// the candidates within the error bound in FP64 (the same top-k as the exact
// path), false returns the split-BF16 scores and their top-k.
uint32_t engine_rankquant_full_split(const Index& rq, const float* d_q, uint64_t nq, uint64_t k, bool exact,
                                     Workspace& w, cudaStream_t st, uint32_t q_per_tile = 0);
// The exact split search with a fixed candidate count kp and no host
// synchronisation (capturable once the workspace is sized; nq * n * 4 bytes of
// keys must fit the key budget): *d_flag |= 1 (caller-zeroed) when the margin
// test fails for some query, i.e. when kp was too small for an exact result.
uint32_t engine_rankquant_split_fixed(const Index& rq, const float* d_q, uint64_t nq, uint64_t k, uint64_t kp,
                                      uint32_t q_per_tile, uint32_t* d_flag, Workspace& w, cudaStream_t st);
uint32_t engine_rankquant_subset(const Index& rq, const float* d_q, uint64_t nq,
                                 const uint64_t* d_off, const uint32_t* d_cands, uint64_t max_row,
                                 uint64_t k, Workspace& w, cudaStream_t st);
// RankQuant::search (symmetric: the query is rank-bucketed like a document)
uint32_t engine_rankquant_symmetric(const Index& rq, const float* d_q, uint64_t nq, uint64_t k, Workspace& w,
                                    cudaStream_t st);
// Rank::search (asymmetric = false) / Rank::search_asymmetric
uint32_t engine_rank_full(const Index& rk, const float* d_q, uint64_t nq, uint64_t k, bool asymmetric, Workspace& w,
                          cudaStream_t st);
uint32_t engine_candidates(const Index& s1, const float* d_q, uint64_t nq, uint64_t m,
                           const float* d_weights, Workspace& w, cudaStream_t st,
                           const float* q_unit = nullptr);
uint32_t engine_bitmap_full(const Index& bm, const float* d_q, uint64_t nq, uint64_t k,
                            Workspace& w, cudaStream_t st);
uint32_t engine_fastscan_full(const Index& fs, const float* d_q, uint64_t nq, uint64_t k,
                              Workspace& w, cudaStream_t st);
uint32_t engine_two_stage(const Index& rq, const Index& s1, const float* d_q, uint64_t nq,
                          uint64_t m, uint64_t k, Workspace& w, cudaStream_t st);
// Two-stage search with its own candidate count per query (m_of[q], each
// already clamped to n): stage 1 selects the ordered top-max(m_of) of every
// query, so query q's own top-m_of[q] is the prefix of its row; the prefixes
// are reranked and each output row holds the top-min(k, m_of[q]) (stride
// min(k, max(m_of)), sentinel padded) -- row q equals a search of query q
// alone with m_of[q] candidates.
uint32_t engine_two_stage_ragged(const Index& rq, const Index& s1, const float* d_q, uint64_t nq,
                                 const uint64_t* m_of, uint64_t k, Workspace& w, cudaStream_t st);
uint64_t default_candidate_count(uint64_t k, uint64_t space);
uint64_t engine_keys_budget();  // bytes a key matrix chunk may take
// Device bytes of a stage-1 top-m's intermediates for nq queries: the sampled
// filter's sample keys and kept rows where a bitmap-family stage 1 takes the
// tensor-core filter, else the key matrix (capped at the chunk budget).
uint64_t engine_stage1_bytes(const Index& s1, uint64_t nq, uint64_t m);
// engine_rankquant_split_fixed can run nq queries of top-k in one chunk
bool split_fixed_fits(const Index& rq, uint64_t nq, uint64_t k);

// mixed batches (mixed.cu): drop the cached plans of an index that is freed or
// grows; plan facts for tests and tools
void mixed_forget_index(const Index* ix);
bool mixed_plan_info(const Index& ix, uint64_t nq, uint64_t k, uint32_t* qpt, uint64_t* kp, uint64_t* replays);

// persistence (persist.cpp)
std::unique_ptr<Index> load_index_file(const char* path, bool v1_only);
void probe_index_file(const char* path, ordvec_index_info_t* info);
void write_index_file(const Index& ix, const char* path);
void read_payload(const Index& ix, std::vector<uint8_t>& out);
void upload_payload(Index& ix, const uint8_t* payload, uint64_t bytes);

extern thread_local uint64_t tl_last_launches;

// C-ABI error boundary (status + thread-local message) for entry points in
// other files; tensor-core error word check after a synchronised pipeline.
ordvec_status_t api_boundary(const std::function<void()>& f);
void check_tc_errors(Workspace& w);

}  // namespace ovb
