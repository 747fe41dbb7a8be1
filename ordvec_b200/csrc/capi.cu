// C ABI of libordvec_b200 (include/ordvec_b200.h).
//
// Part 1 mirrors ordvec-ffi (ordvec-ffi/src/lib.rs): the same status codes,
// thread-local last error, exact struct-size rule, validation order
// (validate_search, :444-568) and result semantics (full search ->
// search_asymmetric / Bitmap::search; subset -> score every candidate then
// order by (score desc, row asc) and truncate, :959-981).  Exceptions never
// cross the boundary: they become statuses the way ffi_boundary turns panics
// into ORDVEC_STATUS_PANIC (:224-239).
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>

#include "ovb_host.h"

namespace ovb {

thread_local uint64_t tl_launch_counter = 0;
thread_local uint64_t tl_last_launches = 0;

namespace {
thread_local std::string tl_error;

template <class F>
ordvec_status_t boundary(F&& f) noexcept {
  tl_launch_counter = 0;
  try {
    f();
    tl_error.clear();
    tl_last_launches = tl_launch_counter;
    return ORDVEC_STATUS_OK;
  } catch (const ApiError& e) {
    tl_error = e.msg;
    return e.status;
  } catch (const CudaError& e) {
    tl_error = e.what();
    return ORDVEC_STATUS_INTERNAL;
  } catch (const std::bad_alloc&) {
    tl_error = "allocation failed";
    return ORDVEC_STATUS_INTERNAL;
  } catch (const std::invalid_argument& e) {
    tl_error = e.what();
    return ORDVEC_STATUS_BAD_ARGUMENT;
  } catch (const std::exception& e) {
    tl_error = e.what();
    return ORDVEC_STATUS_PANIC;
  } catch (...) {
    tl_error = "panic crossing ordvec C ABI";
    return ORDVEC_STATUS_PANIC;
  }
}

void check_exact_size(uint64_t got, size_t expected, const char* what) {
  if (got != expected)
    fail(ORDVEC_STATUS_BAD_STRUCT_SIZE, std::string(what) + ".struct_size must be exactly " +
                                            std::to_string(expected) + ", got " + std::to_string(got));
}

bool all_finite(const float* x, uint64_t count) {
  for (uint64_t i = 0; i < count; i++)
    if (!std::isfinite(x[i])) return false;
  return true;
}

uint32_t encode_kind(uint32_t kind) {
  switch (kind) {
    case ORDVEC_INDEX_KIND_RANK_QUANT: return 0;
    case OVB_INDEX_KIND_SIGN_BITMAP: return 1;
    case ORDVEC_INDEX_KIND_BITMAP: return 2;
    case OVB_INDEX_KIND_FASTSCAN: return 3;
    case OVB_INDEX_KIND_RANK: return 5;
    default: return 4;
  }
}

ordvec_index_info_t info_for(const Index& ix) {
  ordvec_index_info_t info;
  ordvec_index_info_init(&info);
  info.kind = ix.kind;
  info.format_version = 1;
  info.dim = ix.dim;
  info.bit_width = ix.kind == ORDVEC_INDEX_KIND_BITMAP || ix.kind == OVB_INDEX_KIND_SIGN_BITMAP ? 0 : ix.bits;
  info.n_top = ix.kind == ORDVEC_INDEX_KIND_BITMAP ? ix.n_top : 0;
  info.vector_count = ix.n;
  info.bytes_per_vec = ix.ref_bytes_per_vec();
  info.source_file_size_bytes = ix.file_size;
  info.capabilities =
      ORDVEC_CAP_FULL_SEARCH | ORDVEC_CAP_SUBSET_SEARCH | ORDVEC_CAP_STATS | ORDVEC_CAP_ID_EQUALS_ROW_ID;
  return info;
}

// Grow the device code buffer to hold `rows`, keeping existing rows.
void grow_codes(Index& ix, uint64_t rows) {
  const uint64_t need = ix.device_bytes(rows), have = ix.device_bytes(ix.n);
  if (need <= ix.codes.cap) return;
  void* p = nullptr;
  uint64_t cap = need > ix.codes.cap + ix.codes.cap / 2 ? need : ix.codes.cap + ix.codes.cap / 2;
  OVB_CUDA(cudaMalloc(&p, cap));
  if (ix.kind == OVB_INDEX_KIND_FASTSCAN) OVB_CUDA(cudaMemset(p, 0, cap));
  if (have) OVB_CUDA(cudaMemcpy(p, ix.codes.p, have, cudaMemcpyDeviceToDevice));
  if (ix.codes.p) cudaFree(ix.codes.p);
  ix.codes.p = p;
  ix.codes.cap = cap;
}

void add_device_rows(Index& ix, const float* d_vecs, uint64_t n, Workspace& w) {
  if (!n) return;
  if (ix.n + n > kMaxVectors)
    fail(ORDVEC_STATUS_BAD_ARGUMENT, "index would exceed MAX_VECTORS (67108864); had " + std::to_string(ix.n) +
                                         ", adding " + std::to_string(n));
  if (ix.kind == OVB_INDEX_KIND_FASTSCAN && ix.n)
    fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION,
         "FastScan v1: incremental add() not supported (block-32 layout); construct a new index");
  if (ix.kind != OVB_INDEX_KIND_SIGN_BITMAP && ix.dim > kMaxDeviceRankDim)
    fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "device rank transform supports dim <= 16384");
  grow_codes(ix, ix.n + n);
  launch_encode((int)encode_kind(ix.kind), d_vecs, n, ix.dim, ix.bits, ix.n_top, ix.pairs_pad, ix.codes.p, ix.n,
                w.stream);
  OVB_CUDA(cudaStreamSynchronize(w.stream));
  ix.n += n;
}

Index* new_index(uint32_t kind, uint32_t dim, uint32_t bits, uint32_t n_top) {
  ensure_device();
  auto* ix = new Index();
  ix->kind = kind;
  ix->dim = dim;
  ix->bits = bits;
  ix->n_top = n_top;
  if (kind == OVB_INDEX_KIND_FASTSCAN) ix->pairs_pad = fastscan_pairs_pad(dim);
  cudaGetDevice(&ix->device);
  return ix;
}

// Up to this many values the finiteness check runs on the host while the copy
// is in flight (a few microseconds, no device round trip); larger batches are
// checked by a kernel, faster than one host thread.
constexpr uint64_t kHostFiniteMax = 1u << 16;

const float* upload_queries(Workspace& w, const float* q, uint64_t nq, uint32_t dim, bool check) {
  float* d = (float*)w.q_raw.ensure(nq * dim * 4);
  OVB_CUDA(cudaMemcpyAsync(d, q, nq * dim * 4, cudaMemcpyHostToDevice, w.stream));
  if (check && nq * dim <= kHostFiniteMax) {
    if (!all_finite(q, nq * dim)) {
      OVB_CUDA(cudaStreamSynchronize(w.stream));  // the copy still reads the caller's buffer
      fail(ORDVEC_STATUS_NONFINITE_QUERY, "query contains NaN or infinity");
    }
  } else if (check) {
    uint32_t* flag = (uint32_t*)w.flag.ensure(4);
    uint32_t* h = (uint32_t*)w.pinned.ensure(4);
    OVB_CUDA(cudaMemsetAsync(flag, 0, 4, w.stream));
    launch_finite_flag(d, nq * dim, flag, w.stream);
    OVB_CUDA(cudaMemcpyAsync(h, flag, 4, cudaMemcpyDeviceToHost, w.stream));
    OVB_CUDA(cudaStreamSynchronize(w.stream));
    if (*h) fail(ORDVEC_STATUS_NONFINITE_QUERY, "query contains NaN or infinity");
  }
  return d;
}

// After a synchronised pipeline: surface a timed-out wait of a tensor-core
// kernel (its results are then incomplete) as INTERNAL, and re-arm the word.
void check_tc(Workspace& w) {
  if (!w.tc_used) return;
  w.tc_used = false;
  uint32_t* h = (uint32_t*)w.pinned.ensure(4);
  OVB_CUDA(cudaMemcpyAsync(h, w.tc_err.p, 4, cudaMemcpyDeviceToHost, w.stream));
  OVB_CUDA(cudaStreamSynchronize(w.stream));
  if (*h) {
    OVB_CUDA(cudaMemsetAsync(w.tc_err.p, 0, 4, w.stream));
    OVB_CUDA(cudaStreamSynchronize(w.stream));
    fail(ORDVEC_STATUS_INTERNAL, "tensor-core FastScan scan: a bounded wait timed out; results discarded");
  }
}

// results of the last pipeline (w.out_keys / w.out_ids, count entries) -> host
void download_results(Workspace& w, uint64_t count, int mode, uint32_t n_top, float* scores, int64_t* ids) {
  if (!count) return;
  float* ds = (float*)w.scores.ensure(count * 4);
  int64_t* di = (int64_t*)w.ids.ensure(count * 8);
  launch_keys_to_results(w.out_keys.as<uint32_t>(), w.out_ids.as<uint32_t>(), count, mode, n_top, ds, di, w.stream);
  OVB_CUDA(cudaMemcpyAsync(scores, ds, count * 4, cudaMemcpyDeviceToHost, w.stream));
  OVB_CUDA(cudaMemcpyAsync(ids, di, count * 8, cudaMemcpyDeviceToHost, w.stream));
  // the tensor-core error word comes back with the results: one synchronisation
  uint32_t* h_err = w.tc_used ? (uint32_t*)w.pinned.ensure(4) : nullptr;
  if (h_err) OVB_CUDA(cudaMemcpyAsync(h_err, w.tc_err.p, 4, cudaMemcpyDeviceToHost, w.stream));
  OVB_CUDA(cudaStreamSynchronize(w.stream));
  if (h_err) {
    w.tc_used = false;
    if (*h_err) {
      OVB_CUDA(cudaMemsetAsync(w.tc_err.p, 0, 4, w.stream));
      OVB_CUDA(cudaStreamSynchronize(w.stream));
      fail(ORDVEC_STATUS_INTERNAL, "tensor-core FastScan scan: a bounded wait timed out; results discarded");
    }
  }
}

void need_queries(const float* q, uint64_t nq) {
  if (nq && !q) fail(ORDVEC_STATUS_NULL_POINTER, "queries pointer is NULL");
}

// Bitmap subset (src/bitmap.rs:470-494) on one CSR row set.
uint32_t bitmap_subset(const Index& bm, const float* d_q, uint64_t nq, const uint64_t* d_off,
                       const uint32_t* d_cands, uint64_t max_row, uint64_t total, uint64_t k, Workspace& w) {
  const uint32_t ke = (uint32_t)(k < max_row ? k : max_row);
  if (!ke || !nq) return ke;
  uint64_t* qb = (uint64_t*)w.qbits.ensure(nq * bm.qpv() * 8);
  launch_bitmap_query(d_q, nq, bm.dim, bm.n_top, qb, w.stream);
  uint32_t* keys = (uint32_t*)w.keys2.ensure(total * 4);
  launch_popc_subset(1, bm.codes.as<uint64_t>(), bm.qpv(), qb, nq, d_off, d_cands, max_row, bm.n_top, keys,
                     w.stream);
  SelectArgs a{keys, d_cands, d_off, 0, 0, ke, bits_for(bm.n_top), bits_for(bm.n ? bm.n - 1 : 0),
               (uint32_t*)w.out_keys.ensure(nq * ke * 4), (uint32_t*)w.out_ids.ensure(nq * ke * 4)};
  size_t se = select_rows_scratch_elems(nq, ke, 0);
  launch_select_rows(a, nq, se ? (uint64_t*)w.scratch.ensure(se * 8) : nullptr, w.stream);
  return ke;
}

}  // namespace

ordvec_status_t api_boundary(const std::function<void()>& f) { return boundary(f); }
void check_tc_errors(Workspace& w) { check_tc(w); }

Workspace::Workspace() {
  OVB_CUDA(cudaGetDevice(&device));
  OVB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
}
Workspace::~Workspace() {
  if (stream) cudaStreamDestroy(stream);
}

void ensure_device() {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION,
         std::string("no CUDA device available: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "0 devices"));
  }
}

Workspace& workspace() {
  thread_local std::unique_ptr<Workspace> w;
  ensure_device();
  int dev = 0;
  OVB_CUDA(cudaGetDevice(&dev));
  if (!w || w->device != dev) w.reset(new Workspace());
  return *w;
}

const Index& as_index(const ordvec_index_t* h) {
  if (!h) fail(ORDVEC_STATUS_NULL_POINTER, "index pointer is NULL");
  const Index* ix = (const Index*)h;
  if (ix->magic != kIndexMagic) fail(ORDVEC_STATUS_BAD_ARGUMENT, "not a live ordvec index handle");
  return *ix;
}
Index& as_index_mut(ordvec_index_t* h) { return const_cast<Index&>(as_index(h)); }

}  // namespace ovb

using namespace ovb;

extern "C" {

/* ---------------- Part 1: ordvec C ABI v1 ---------------- */

uint32_t ordvec_abi_version(void) { return ORDVEC_ABI_VERSION; }

const char* ordvec_version_string(void) { return "0.6.0+b200"; }

const char* ordvec_status_name(ordvec_status_t s) {
  switch (s) {
    case ORDVEC_STATUS_OK: return "OK";
    case ORDVEC_STATUS_NULL_POINTER: return "NULL_POINTER";
    case ORDVEC_STATUS_BAD_ARGUMENT: return "BAD_ARGUMENT";
    case ORDVEC_STATUS_BAD_STRUCT_SIZE: return "BAD_STRUCT_SIZE";
    case ORDVEC_STATUS_UNSUPPORTED_FORMAT: return "UNSUPPORTED_FORMAT";
    case ORDVEC_STATUS_CORRUPT_INDEX: return "CORRUPT_INDEX";
    case ORDVEC_STATUS_IO: return "IO";
    case ORDVEC_STATUS_DIM_MISMATCH: return "DIM_MISMATCH";
    case ORDVEC_STATUS_NONFINITE_QUERY: return "NONFINITE_QUERY";
    case ORDVEC_STATUS_ROW_ID_OUT_OF_RANGE: return "ROW_ID_OUT_OF_RANGE";
    case ORDVEC_STATUS_BUFFER_TOO_SMALL: return "BUFFER_TOO_SMALL";
    case ORDVEC_STATUS_UNSUPPORTED_OPERATION: return "UNSUPPORTED_OPERATION";
    case ORDVEC_STATUS_PANIC: return "PANIC";
    case ORDVEC_STATUS_INTERNAL: return "INTERNAL";
    default: return "UNKNOWN";
  }
}

const char* ordvec_last_error(void) { return tl_error.c_str(); }

ordvec_status_t ordvec_init(void) {
  return boundary([] {
    ensure_device();
    OVB_CUDA(cudaFree(nullptr));
  });
}

void ordvec_index_info_init(ordvec_index_info_t* info) {
  if (!info) return;
  memset(info, 0, sizeof(*info));
  info->struct_size = sizeof(ordvec_index_info_t);
}

void ordvec_search_params_init(ordvec_search_params_t* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->struct_size = sizeof(ordvec_search_params_t);
}

void ordvec_search_stats_init(ordvec_search_stats_t* s) {
  if (!s) return;
  memset(s, 0, sizeof(*s));
  s->struct_size = sizeof(ordvec_search_stats_t);
  s->abi_version = ORDVEC_ABI_VERSION;
}

ordvec_status_t ordvec_index_load(const char* path, uint64_t flags, ordvec_index_t** out) {
  return boundary([&] {
    if (!path) fail(ORDVEC_STATUS_NULL_POINTER, "path pointer is NULL");
    if (!out) fail(ORDVEC_STATUS_NULL_POINTER, "out pointer is NULL");
    *out = nullptr;
    if (flags) fail(ORDVEC_STATUS_BAD_ARGUMENT, "unknown load flags: " + std::to_string(flags));
    *out = (ordvec_index_t*)load_index_file(path, true).release();
  });
}

ordvec_status_t ordvec_index_probe(const char* path, uint64_t flags, ordvec_index_info_t* info_out) {
  return boundary([&] {
    if (!path) fail(ORDVEC_STATUS_NULL_POINTER, "path pointer is NULL");
    if (!info_out) fail(ORDVEC_STATUS_NULL_POINTER, "info_out pointer is NULL");
    if (flags) fail(ORDVEC_STATUS_BAD_ARGUMENT, "unknown probe flags: " + std::to_string(flags));
    check_exact_size(info_out->struct_size, sizeof(ordvec_index_info_t), "ordvec_index_info_t");
    ordvec_index_info_t info;
    probe_index_file(path, &info);
    *info_out = info;
  });
}

ordvec_status_t ordvec_index_info(const ordvec_index_t* index, ordvec_index_info_t* info_out) {
  return boundary([&] {
    const Index& ix = as_index(index);
    if (!info_out) fail(ORDVEC_STATUS_NULL_POINTER, "info_out pointer is NULL");
    check_exact_size(info_out->struct_size, sizeof(ordvec_index_info_t), "ordvec_index_info_t");
    *info_out = info_for(ix);
  });
}

void ordvec_index_free(ordvec_index_t* index) {
  if (!index) return;
  Index* ix = (Index*)index;
  if (ix->magic != kIndexMagic) return;
  mixed_forget_index(ix);
  ix->magic = 0;
  delete ix;
}

ordvec_status_t ordvec_index_search(const ordvec_index_t* index, const ordvec_search_params_t* params,
                                    ordvec_hit_t* hits_out, uint64_t hits_capacity, uint64_t* returned_out,
                                    ordvec_search_stats_t* stats_out) {
  return boundary([&] {
    const auto started = std::chrono::steady_clock::now();
    const Index& ix = as_index(index);
    if (!params) fail(ORDVEC_STATUS_NULL_POINTER, "params pointer is NULL");
    const ordvec_search_params_t& p = *params;
    // validate_search (ordvec-ffi/src/lib.rs:444-568), same order
    check_exact_size(p.struct_size, sizeof(ordvec_search_params_t), "ordvec_search_params_t");
    if (p.flags != ORDVEC_SEARCH_FLAG_NONE)
      fail(ORDVEC_STATUS_BAD_ARGUMENT, "unknown search flags: " + std::to_string(p.flags));
    for (int i = 0; i < 8; i++)
      if (p.reserved[i]) fail(ORDVEC_STATUS_BAD_ARGUMENT, "ordvec_search_params_t.reserved fields must be zero");
    if (!returned_out) fail(ORDVEC_STATUS_NULL_POINTER, "returned_out pointer is NULL");
    if (stats_out) check_exact_size(stats_out->struct_size, sizeof(ordvec_search_stats_t), "ordvec_search_stats_t");
    if (!p.query) fail(ORDVEC_STATUS_NULL_POINTER, "query pointer is NULL");
    if (p.dim != ix.dim)
      fail(ORDVEC_STATUS_DIM_MISMATCH,
           "query dim " + std::to_string(p.dim) + " does not match index dim " + std::to_string(ix.dim));
    if (!all_finite(p.query, ix.dim)) fail(ORDVEC_STATUS_NONFINITE_QUERY, "query contains NaN or infinity");
    const uint32_t* rows = nullptr;
    if (p.candidate_count == 0 && p.candidate_rows)
      fail(ORDVEC_STATUS_BAD_ARGUMENT, "candidate_count is zero but candidate_rows is non-NULL");
    if (p.candidate_count && !p.candidate_rows)
      fail(ORDVEC_STATUS_NULL_POINTER, "candidate_rows pointer is NULL but candidate_count is nonzero");
    if (p.candidate_count) {
      rows = p.candidate_rows;
      for (uint64_t i = 0; i < p.candidate_count; i++)
        if (rows[i] >= ix.n)
          fail(ORDVEC_STATUS_ROW_ID_OUT_OF_RANGE, "candidate row " + std::to_string(rows[i]) +
                                                       " is out of range for " + std::to_string(ix.n) + " vectors");
    }
    const uint64_t space = rows ? p.candidate_count : ix.n;
    const uint64_t required = p.k < space ? p.k : space;
    if (required) {
      if (!hits_out) fail(ORDVEC_STATUS_NULL_POINTER, "hits_out pointer is NULL");
      if (hits_capacity < required)
        fail(ORDVEC_STATUS_BUFFER_TOO_SMALL, "hits_capacity " + std::to_string(hits_capacity) +
                                                 " is smaller than required " + std::to_string(required));
    }
    if (ix.kind != ORDVEC_INDEX_KIND_RANK_QUANT && ix.kind != ORDVEC_INDEX_KIND_BITMAP)
      fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "ABI v1 searches only RankQuant and Bitmap indexes");
    uint64_t returned = 0;
    if (required) {
      if (ix.kind == ORDVEC_INDEX_KIND_RANK_QUANT && rows && p.candidate_count > ix.n)
        fail(ORDVEC_STATUS_PANIC, "search_asymmetric_subset: candidate list length " +
                                      std::to_string(p.candidate_count) + " exceeds n_vectors " +
                                      std::to_string(ix.n) + "; deduplicate repeated ids before calling");
      Workspace& w = workspace();
      const float* d_q = upload_queries(w, p.query, 1, ix.dim, false);
      uint32_t ke = 0;
      if (!rows) {
        ke = ix.kind == ORDVEC_INDEX_KIND_RANK_QUANT ? engine_rankquant_full(ix, d_q, 1, required, w, w.stream)
                                                     : engine_bitmap_full(ix, d_q, 1, required, w, w.stream);
      } else {
        uint64_t hoff[2] = {0, p.candidate_count};
        uint64_t* d_off = (uint64_t*)w.off.ensure(16);
        uint32_t* d_c = (uint32_t*)w.sel_ids.ensure(p.candidate_count * 4);
        OVB_CUDA(cudaMemcpyAsync(d_off, hoff, 16, cudaMemcpyHostToDevice, w.stream));
        OVB_CUDA(cudaMemcpyAsync(d_c, rows, p.candidate_count * 4, cudaMemcpyHostToDevice, w.stream));
        ke = ix.kind == ORDVEC_INDEX_KIND_RANK_QUANT
                 ? engine_rankquant_subset(ix, d_q, 1, d_off, d_c, p.candidate_count, required, w, w.stream)
                 : bitmap_subset(ix, d_q, 1, d_off, d_c, p.candidate_count, p.candidate_count, required, w);
      }
      std::vector<float> sc(ke);
      std::vector<int64_t> id(ke);
      download_results(w, ke, ix.kind == ORDVEC_INDEX_KIND_RANK_QUANT ? 0 : 1, ix.n_top, sc.data(), id.data());
      for (uint32_t s = 0; s < ke; s++) {
        if (id[s] < 0) break;
        hits_out[s].row_id = (uint64_t)id[s];
        hits_out[s].id = (uint64_t)id[s];
        hits_out[s].score = sc[s];
        hits_out[s].reserved = 0;
        returned++;
      }
    }
    *returned_out = returned;
    if (stats_out) {
      ordvec_search_stats_t st;
      ordvec_search_stats_init(&st);
      st.kind = ix.kind;
      st.dim = ix.dim;
      st.bit_width = ix.kind == ORDVEC_INDEX_KIND_RANK_QUANT ? ix.bits : 0;
      st.n_top = ix.kind == ORDVEC_INDEX_KIND_BITMAP ? ix.n_top : 0;
      st.k = p.k;
      st.user_tag = p.user_tag;
      st.vector_count = ix.n;
      st.candidate_count = space;
      st.returned_count = returned;
      st.total_ns = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                        std::chrono::steady_clock::now() - started)
                        .count();
      st.vectors_scored = space;
      *stats_out = st;
    }
  });
}

/* ---------------- Part 2: extensions ---------------- */

ordvec_status_t ovb_rankquant_new(uint32_t dim, uint32_t bits, ordvec_index_t** out) {
  return boundary([&] {
    if (!out) fail(ORDVEC_STATUS_NULL_POINTER, "out pointer is NULL");
    *out = nullptr;
    // RankQuant::validate_params (src/quant.rs:375-420)
    if (bits != 1 && bits != 2 && bits != 4 && bits != 8)
      fail(ORDVEC_STATUS_BAD_ARGUMENT, "bits: must be 1, 2, 4, or 8");
    if (dim < 2) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim: must be >= 2");
    if (dim > 65535) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim: must fit in u16");
    if (dim % (8 / bits)) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim: must be a multiple of codes per byte");
    if (bits == 8) fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "b=8 RankQuant has no device path");
    if (dim % (1u << bits)) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim: must be divisible by 2^bits");
    *out = (ordvec_index_t*)new_index(ORDVEC_INDEX_KIND_RANK_QUANT, dim, bits, 0);
  });
}

ordvec_status_t ovb_sign_bitmap_new(uint32_t dim, ordvec_index_t** out) {
  return boundary([&] {
    if (!out) fail(ORDVEC_STATUS_NULL_POINTER, "out pointer is NULL");
    *out = nullptr;
    // SignBitmap::validate_dim (src/sign_bitmap.rs:113-136)
    if (dim == 0) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim: must be > 0");
    if (dim % 64) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim: must be a multiple of 64");
    if (dim > kMaxSignDim) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim: must be <= MAX_SIGN_BITMAP_DIM");
    *out = (ordvec_index_t*)new_index(OVB_INDEX_KIND_SIGN_BITMAP, dim, 1, 0);
  });
}

ordvec_status_t ovb_bitmap_new(uint32_t dim, uint32_t n_top, ordvec_index_t** out) {
  return boundary([&] {
    if (!out) fail(ORDVEC_STATUS_NULL_POINTER, "out pointer is NULL");
    *out = nullptr;
    // Bitmap::validate_params (src/bitmap.rs:71-100)
    if (dim == 0) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim: must be > 0");
    if (dim % 64) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim: must be a multiple of 64");
    if (dim > kMaxDim) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim: must be <= 65535 (u16 rank invariant)");
    if (!(n_top > 0 && n_top < dim)) fail(ORDVEC_STATUS_BAD_ARGUMENT, "n_top: must satisfy 0 < n_top < dim");
    *out = (ordvec_index_t*)new_index(ORDVEC_INDEX_KIND_BITMAP, dim, 0, n_top);
  });
}

ordvec_status_t ovb_fastscan_new(uint32_t dim, ordvec_index_t** out) {
  return boundary([&] {
    if (!out) fail(ORDVEC_STATUS_NULL_POINTER, "out pointer is NULL");
    *out = nullptr;
    // RankQuantFastscan::new (src/fastscan.rs:568-589)
    if (dim < 2) fail(ORDVEC_STATUS_BAD_ARGUMENT, "FastScan b=2: dim must be >= 2");
    if (dim > 65535) fail(ORDVEC_STATUS_BAD_ARGUMENT, "FastScan b=2: dim must fit in u16");
    if (dim % 4) fail(ORDVEC_STATUS_BAD_ARGUMENT, "FastScan b=2: dim must be divisible by 4");
    *out = (ordvec_index_t*)new_index(OVB_INDEX_KIND_FASTSCAN, dim, 2, 0);
  });
}

ordvec_status_t ovb_multibucket_new(uint32_t dim, uint32_t bits, ordvec_index_t** out) {
  return boundary([&] {
    if (!out) fail(ORDVEC_STATUS_NULL_POINTER, "out pointer is NULL");
    *out = nullptr;
    // MultiBucketBitmap::new (src/multi_bucket.rs:70-93)
    if (bits != 1 && bits != 2 && bits != 4) fail(ORDVEC_STATUS_BAD_ARGUMENT, "bits must be 1, 2, or 4");
    if (dim == 0) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim must be > 0");
    if (dim % 64) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim must be a multiple of 64");
    if (dim % (1u << bits)) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim must be a multiple of 2^bits");
    if (dim > kMaxDim) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim must be <= 65535");
    *out = (ordvec_index_t*)new_index(OVB_INDEX_KIND_MULTIBUCKET, dim, bits, 0);
  });
}

ordvec_status_t ovb_rank_new(uint32_t dim, ordvec_index_t** out) {
  return boundary([&] {
    if (!out) fail(ORDVEC_STATUS_NULL_POINTER, "out pointer is NULL");
    *out = nullptr;
    // Rank::new (src/rank.rs:316-324)
    if (dim < 2) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim must be >= 2");
    if (dim > 65535) fail(ORDVEC_STATUS_BAD_ARGUMENT, "dim must fit in u16");
    *out = (ordvec_index_t*)new_index(OVB_INDEX_KIND_RANK, dim, 16, 0);
  });
}

ordvec_status_t ovb_index_add(ordvec_index_t* index, const float* vectors, uint64_t n) {
  return boundary([&] {
    Index& ix = as_index_mut(index);
    mixed_forget_index(&ix);  // cached mixed-batch plans describe the old rows
    if (n && !vectors) fail(ORDVEC_STATUS_NULL_POINTER, "vectors pointer is NULL");
    if (!n) return;
    if (!all_finite(vectors, n * ix.dim))
      fail(ORDVEC_STATUS_BAD_ARGUMENT, "ordvec: input contains non-finite (NaN or +-Inf) values; embeddings must be finite");
    Workspace& w = workspace();
    const uint64_t chunk = ((256ull << 20) / (ix.dim * 4ull)) & ~31ull;
    const uint64_t step = chunk ? chunk : 32;
    for (uint64_t r0 = 0; r0 < n; r0 += step) {
      const uint64_t rn = n - r0 < step ? n - r0 : step;
      float* d = (float*)w.stage.ensure(rn * ix.dim * 4);
      OVB_CUDA(cudaMemcpyAsync(d, vectors + r0 * ix.dim, rn * ix.dim * 4, cudaMemcpyHostToDevice, w.stream));
      if (ix.kind == OVB_INDEX_KIND_FASTSCAN && r0 == 0 && rn < n) {
        // FastScan is single-shot: stage the whole corpus through device memory
        float* all = nullptr;
        OVB_CUDA(cudaMalloc(&all, n * ix.dim * 4));
        OVB_CUDA(cudaMemcpy(all, vectors, n * ix.dim * 4, cudaMemcpyHostToDevice));
        try {
          add_device_rows(ix, all, n, w);
        } catch (...) {
          cudaFree(all);
          throw;
        }
        cudaFree(all);
        return;
      }
      add_device_rows(ix, d, rn, w);
    }
  });
}

ordvec_status_t ovb_index_add_device(ordvec_index_t* index, const float* d_vectors, uint64_t n) {
  return boundary([&] {
    Index& ix = as_index_mut(index);
    mixed_forget_index(&ix);  // cached mixed-batch plans describe the old rows
    if (n && !d_vectors) fail(ORDVEC_STATUS_NULL_POINTER, "vectors pointer is NULL");
    if (!n) return;
    Workspace& w = workspace();
    uint32_t* flag = (uint32_t*)w.flag.ensure(4);
    uint32_t* h = (uint32_t*)w.pinned.ensure(4);
    OVB_CUDA(cudaMemsetAsync(flag, 0, 4, w.stream));
    launch_finite_flag(d_vectors, n * ix.dim, flag, w.stream);
    OVB_CUDA(cudaMemcpyAsync(h, flag, 4, cudaMemcpyDeviceToHost, w.stream));
    OVB_CUDA(cudaStreamSynchronize(w.stream));
    if (*h) fail(ORDVEC_STATUS_BAD_ARGUMENT, "ordvec: input contains non-finite (NaN or +-Inf) values");
    add_device_rows(ix, d_vectors, n, w);
  });
}

ordvec_status_t ovb_index_load_any(const char* path, uint64_t flags, ordvec_index_t** out) {
  return boundary([&] {
    if (!path) fail(ORDVEC_STATUS_NULL_POINTER, "path pointer is NULL");
    if (!out) fail(ORDVEC_STATUS_NULL_POINTER, "out pointer is NULL");
    *out = nullptr;
    if (flags) fail(ORDVEC_STATUS_BAD_ARGUMENT, "unknown load flags: " + std::to_string(flags));
    *out = (ordvec_index_t*)load_index_file(path, false).release();
  });
}

ordvec_status_t ovb_index_write(const ordvec_index_t* index, const char* path) {
  return boundary([&] {
    const Index& ix = as_index(index);
    if (!path) fail(ORDVEC_STATUS_NULL_POINTER, "path pointer is NULL");
    write_index_file(ix, path);
  });
}

ordvec_status_t ovb_index_payload_bytes(const ordvec_index_t* index, uint64_t* bytes_out) {
  return boundary([&] {
    const Index& ix = as_index(index);
    if (!bytes_out) fail(ORDVEC_STATUS_NULL_POINTER, "bytes_out pointer is NULL");
    *bytes_out = ix.kind == OVB_INDEX_KIND_FASTSCAN ? ((ix.n + 31) / 32) * (uint64_t)(ix.dim / 2) * 32
                                                    : ix.device_bytes(ix.n);
  });
}

ordvec_status_t ovb_index_payload(const ordvec_index_t* index, void* out, uint64_t bytes) {
  return boundary([&] {
    const Index& ix = as_index(index);
    std::vector<uint8_t> p;
    read_payload(ix, p);
    if (bytes < p.size()) fail(ORDVEC_STATUS_BUFFER_TOO_SMALL, "payload buffer too small");
    if (!out && !p.empty()) fail(ORDVEC_STATUS_NULL_POINTER, "out pointer is NULL");
    if (!p.empty()) memcpy(out, p.data(), p.size());
  });
}

ordvec_status_t ovb_rankquant_search(const ordvec_index_t* rq, const float* queries, uint64_t nq, uint64_t k,
                                     float* scores, int64_t* ids) {
  return boundary([&] {
    const Index& ix = as_index(rq);
    need_queries(queries, nq);
    const uint64_t ke = k < ix.n ? k : ix.n;
    if (!ke || !nq) return;
    if (!scores || !ids) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    Workspace& w = workspace();
    const float* d_q = upload_queries(w, queries, nq, ix.dim, true);
    uint32_t got = engine_rankquant_full(ix, d_q, nq, ke, w, w.stream);
    download_results(w, nq * got, 0, 0, scores, ids);
  });
}

ordvec_status_t ovb_rankquant_search_split(const ordvec_index_t* rq, const float* queries, uint64_t nq, uint64_t k,
                                           uint32_t exact, float* scores, int64_t* ids) {
  return boundary([&] {
    const Index& ix = as_index(rq);
    need_queries(queries, nq);
    const uint64_t ke = k < ix.n ? k : ix.n;
    if (!ke || !nq) return;
    if (!scores || !ids) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    Workspace& w = workspace();
    const float* d_q = upload_queries(w, queries, nq, ix.dim, true);
    uint32_t got = engine_rankquant_full_split(ix, d_q, nq, ke, exact != 0, w, w.stream);
    download_results(w, nq * got, 0, 0, scores, ids);
  });
}

ordvec_status_t ovb_rankquant_search_subset(const ordvec_index_t* rq, const float* queries, uint64_t nq,
                                            const uint64_t* offsets, const uint32_t* candidates, uint64_t k,
                                            float* scores, int64_t* ids) {
  return boundary([&] {
    const Index& ix = as_index(rq);
    need_queries(queries, nq);
    if (!offsets) fail(ORDVEC_STATUS_NULL_POINTER, "offsets pointer is NULL");
    // validate_csr_batch (src/quant.rs:1088-1119)
    if (offsets[0] != 0) fail(ORDVEC_STATUS_BAD_ARGUMENT, "candidate_offsets[0] must be 0");
    uint64_t max_row = 0;
    for (uint64_t q = 0; q < nq; q++) {
      if (offsets[q + 1] < offsets[q])
        fail(ORDVEC_STATUS_BAD_ARGUMENT, "candidate_offsets must be monotonic non-decreasing");
      const uint64_t len = offsets[q + 1] - offsets[q];
      if (len > ix.n)
        fail(ORDVEC_STATUS_BAD_ARGUMENT, "per-row candidate count " + std::to_string(len) + " exceeds n_vectors " +
                                             std::to_string(ix.n));
      if (len > max_row) max_row = len;
    }
    const uint64_t total = offsets[nq];
    if (total && !candidates) fail(ORDVEC_STATUS_NULL_POINTER, "candidates pointer is NULL");
    for (uint64_t i = 0; i < total; i++)
      if (candidates[i] >= ix.n)
        fail(ORDVEC_STATUS_ROW_ID_OUT_OF_RANGE, "candidate id out of range (n_vectors " + std::to_string(ix.n) + ")");
    const uint64_t ke = k < ix.n ? k : ix.n;
    if (!ke || !nq) return;
    if (!scores || !ids) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    Workspace& w = workspace();
    const float* d_q = upload_queries(w, queries, nq, ix.dim, true);
    uint64_t* d_off = (uint64_t*)w.off.ensure((nq + 1) * 8);
    uint32_t* d_c = (uint32_t*)w.sel_ids.ensure((total ? total : 1) * 4);
    OVB_CUDA(cudaMemcpyAsync(d_off, offsets, (nq + 1) * 8, cudaMemcpyHostToDevice, w.stream));
    if (total) OVB_CUDA(cudaMemcpyAsync(d_c, candidates, total * 4, cudaMemcpyHostToDevice, w.stream));
    uint32_t got = engine_rankquant_subset(ix, d_q, nq, d_off, d_c, max_row, ke, w, w.stream);
    download_results(w, nq * got, 0, 0, scores, ids);
  });
}

static void top_m_host(const Index& ix, const float* queries, uint64_t nq, uint64_t m, const float* weights,
                       uint32_t* out) {
  need_queries(queries, nq);
  const uint64_t me = m < ix.n ? m : ix.n;
  if (!me || !nq) return;
  if (!out) fail(ORDVEC_STATUS_NULL_POINTER, "candidates pointer is NULL");
  Workspace& w = workspace();
  const float* d_q = upload_queries(w, queries, nq, ix.dim, true);
  const float* d_w = nullptr;
  bool identity = weights != nullptr;  // identity weights take the integer (tensor-core) path
  for (uint32_t a = 0; identity && a < ix.nb(); a++)
    for (uint32_t b = 0; b < ix.nb(); b++)
      if (weights[a * ix.nb() + b] != (a == b ? 1.0f : 0.0f)) identity = false;
  if (weights && !identity) {
    float* dw = (float*)w.weights.ensure(ix.nb() * ix.nb() * 4);
    OVB_CUDA(cudaMemcpyAsync(dw, weights, ix.nb() * ix.nb() * 4, cudaMemcpyHostToDevice, w.stream));
    d_w = dw;
  }
  uint32_t got = engine_candidates(ix, d_q, nq, me, d_w, w, w.stream);
  OVB_CUDA(cudaMemcpyAsync(out, w.sel_ids.p, nq * got * 4, cudaMemcpyDeviceToHost, w.stream));
  OVB_CUDA(cudaStreamSynchronize(w.stream));
  check_tc(w);
}

ordvec_status_t ovb_sign_bitmap_top_m(const ordvec_index_t* sign, const float* queries, uint64_t nq, uint64_t m,
                                      uint32_t* candidates) {
  return boundary([&] {
    const Index& ix = as_index(sign);
    if (ix.kind != OVB_INDEX_KIND_SIGN_BITMAP) fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "not a SignBitmap index");
    top_m_host(ix, queries, nq, m, nullptr, candidates);
  });
}

ordvec_status_t ovb_sign_bitmap_score_all(const ordvec_index_t* sign, const float* query, uint32_t* scores) {
  return boundary([&] {
    const Index& ix = as_index(sign);
    if (ix.kind != OVB_INDEX_KIND_SIGN_BITMAP) fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "not a SignBitmap index");
    need_queries(query, 1);
    if (!ix.n) return;
    if (!scores) fail(ORDVEC_STATUS_NULL_POINTER, "scores pointer is NULL");
    Workspace& w = workspace();
    const float* d_q = upload_queries(w, query, 1, ix.dim, true);
    uint64_t* qb = (uint64_t*)w.qbits.ensure(ix.qpv() * 8);
    launch_sign_query(d_q, 1, ix.dim, qb, w.stream);
    uint32_t* keys = (uint32_t*)w.keys.ensure(ix.n * 4);
    launch_popc_scan(0, ix.codes.as<uint64_t>(), ix.n, ix.qpv(), qb, 1, 0, keys, ix.n, w.stream);
    OVB_CUDA(cudaMemcpyAsync(scores, keys, ix.n * 4, cudaMemcpyDeviceToHost, w.stream));
    OVB_CUDA(cudaStreamSynchronize(w.stream));
    for (uint64_t i = 0; i < ix.n; i++) scores[i] = ix.dim - scores[i];
  });
}

ordvec_status_t ovb_bitmap_search(const ordvec_index_t* bm, const float* queries, uint64_t nq, uint64_t k,
                                  float* scores, int64_t* ids) {
  return boundary([&] {
    const Index& ix = as_index(bm);
    need_queries(queries, nq);
    const uint64_t ke = k < ix.n ? k : ix.n;
    if (!ke || !nq) return;
    if (!scores || !ids) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    Workspace& w = workspace();
    const float* d_q = upload_queries(w, queries, nq, ix.dim, true);
    uint32_t got = engine_bitmap_full(ix, d_q, nq, ke, w, w.stream);
    download_results(w, nq * got, 1, ix.n_top, scores, ids);
  });
}

ordvec_status_t ovb_bitmap_top_m(const ordvec_index_t* bm, const float* queries, uint64_t nq, uint64_t m,
                                 uint32_t* candidates) {
  return boundary([&] {
    const Index& ix = as_index(bm);
    if (ix.kind != ORDVEC_INDEX_KIND_BITMAP) fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "not a Bitmap index");
    top_m_host(ix, queries, nq, m, nullptr, candidates);
  });
}

ordvec_status_t ovb_fastscan_search(const ordvec_index_t* fs, const float* queries, uint64_t nq, uint64_t k,
                                    float* scores, int64_t* ids) {
  return boundary([&] {
    const Index& ix = as_index(fs);
    need_queries(queries, nq);
    const uint64_t ke = k < ix.n ? k : ix.n;
    if (!ke || !nq) return;
    if (!scores || !ids) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    Workspace& w = workspace();
    const float* d_q = upload_queries(w, queries, nq, ix.dim, true);
    uint32_t got = engine_fastscan_full(ix, d_q, nq, ke, w, w.stream);
    download_results(w, nq * got, 0, 0, scores, ids);
  });
}

// Full searches whose query is rank-transformed on the device.
static void rank_query_search(const ordvec_index_t* h, uint32_t kind, const char* what, const float* queries,
                              uint64_t nq, uint64_t k, float* scores, int64_t* ids, int variant) {
  const Index& ix = as_index(h);
  if (ix.kind != kind) fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, std::string("not a ") + what + " index");
  need_queries(queries, nq);
  const uint64_t ke = k < ix.n ? k : ix.n;
  if (!ke || !nq) return;
  if (!scores || !ids) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
  if (ix.dim > kMaxDeviceRankDim)  // the rank transform and the scans' shared-memory query row
    fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "device rank search supports dim <= 16384");
  Workspace& w = workspace();
  const float* d_q = upload_queries(w, queries, nq, ix.dim, true);
  uint32_t got = variant == 2 ? engine_rankquant_symmetric(ix, d_q, nq, ke, w, w.stream)
                              : engine_rank_full(ix, d_q, nq, ke, variant == 1, w, w.stream);
  download_results(w, nq * got, 0, 0, scores, ids);
}

ordvec_status_t ovb_rank_search(const ordvec_index_t* rank, const float* queries, uint64_t nq, uint64_t k,
                                float* scores, int64_t* ids) {
  return boundary([&] { rank_query_search(rank, OVB_INDEX_KIND_RANK, "Rank", queries, nq, k, scores, ids, 0); });
}

ordvec_status_t ovb_rank_search_asymmetric(const ordvec_index_t* rank, const float* queries, uint64_t nq,
                                           uint64_t k, float* scores, int64_t* ids) {
  return boundary([&] { rank_query_search(rank, OVB_INDEX_KIND_RANK, "Rank", queries, nq, k, scores, ids, 1); });
}

ordvec_status_t ovb_rankquant_search_symmetric(const ordvec_index_t* rq, const float* queries, uint64_t nq,
                                               uint64_t k, float* scores, int64_t* ids) {
  return boundary([&] {
    rank_query_search(rq, ORDVEC_INDEX_KIND_RANK_QUANT, "RankQuant", queries, nq, k, scores, ids, 2);
  });
}

ordvec_status_t ovb_multibucket_top_m(const ordvec_index_t* mb, const float* queries, uint64_t nq,
                                      const float* weights, uint64_t m, uint32_t* candidates) {
  return boundary([&] {
    const Index& ix = as_index(mb);
    if (ix.kind != OVB_INDEX_KIND_MULTIBUCKET) fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "not a MultiBucketBitmap");
    if (weights)
      for (uint32_t i = 0; i < ix.nb() * ix.nb(); i++)
        if (!std::isfinite(weights[i])) fail(ORDVEC_STATUS_BAD_ARGUMENT, "weights must be finite");
    top_m_host(ix, queries, nq, m, weights, candidates);
  });
}

ordvec_status_t ovb_two_stage_search(const ordvec_index_t* rq, const ordvec_index_t* stage1, const float* queries,
                                     uint64_t nq, uint64_t m, uint64_t k, float* scores, int64_t* ids) {
  return boundary([&] {
    const Index& r = as_index(rq);
    const Index& s = as_index(stage1);
    need_queries(queries, nq);
    if (!nq || !k || !r.n) return;
    if (!scores || !ids) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    Workspace& w = workspace();
    const float* d_q = upload_queries(w, queries, nq, r.dim, true);
    uint32_t got = engine_two_stage(r, s, d_q, nq, m, k, w, w.stream);
    download_results(w, nq * got, 0, 0, scores, ids);
  });
}

ordvec_status_t ovb_two_stage_search_device(const ordvec_index_t* rq, const ordvec_index_t* stage1,
                                            const float* d_queries, uint64_t nq, uint64_t m, uint64_t k,
                                            float* d_scores, int64_t* d_ids, void* stream) {
  return boundary([&] {
    const Index& r = as_index(rq);
    const Index& s = as_index(stage1);
    need_queries(d_queries, nq);
    if (!nq || !k || !r.n) return;
    if (!d_scores || !d_ids) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    Workspace& w = workspace();
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t got = engine_two_stage(r, s, d_queries, nq, m, k, w, st);
    launch_keys_to_results(w.out_keys.as<uint32_t>(), w.out_ids.as<uint32_t>(), nq * got, 0, 0, d_scores, d_ids, st);
  });
}

ordvec_status_t ovb_two_stage_search_device_ex(const ordvec_index_t* rq, const ordvec_index_t* stage1,
                                               const float* d_queries, uint64_t nq, uint64_t m, uint64_t k,
                                               float* d_scores, int64_t* d_ids, void* stream, uint32_t rerank_mode) {
  return boundary([&] {
    if (rerank_mode > OVB_RERANK_SPLIT_RAW) fail(ORDVEC_STATUS_BAD_ARGUMENT, "unknown rerank mode");
    const Index& r = as_index(rq);
    const Index& s = as_index(stage1);
    need_queries(d_queries, nq);
    if (!nq || !k || !r.n) return;
    if (!d_scores || !d_ids) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    Workspace& w = workspace();
    cudaStream_t st = (cudaStream_t)stream;
    struct Mode {
      Workspace& w;
      Mode(Workspace& ws, uint32_t m_) : w(ws) { w.rerank_mode = m_; }
      ~Mode() { w.rerank_mode = OVB_RERANK_AUTO; }
    } guard(w, rerank_mode);
    uint32_t got = engine_two_stage(r, s, d_queries, nq, m, k, w, st);
    launch_keys_to_results(w.out_keys.as<uint32_t>(), w.out_ids.as<uint32_t>(), nq * got, 0, 0, d_scores, d_ids, st);
  });
}

ordvec_status_t ovb_selftest_bounded_wait(uint32_t* timed_out, uint64_t* waited_ns) {
  return boundary([&] {
    if (!timed_out || !waited_ns) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    Workspace& w = workspace();
    uint32_t* d = (uint32_t*)w.flag.ensure(16);
    uint32_t* h = (uint32_t*)w.pinned.ensure(16);
    launch_wait_probe(d, w.stream);
    OVB_CUDA(cudaMemcpyAsync(h, d, 12, cudaMemcpyDeviceToHost, w.stream));
    OVB_CUDA(cudaStreamSynchronize(w.stream));
    *timed_out = h[0];
    *waited_ns = (uint64_t)h[1] | ((uint64_t)h[2] << 32);
  });
}

ordvec_status_t ovb_selftest_arm_tc_error(void) {
  return boundary([&] {
    Workspace& w = workspace();
    uint32_t* e = w.tc_err_word(w.stream);
    w.tc_used = false;  // only armed: the next search that runs a tensor-core kernel reads it
    OVB_CUDA(cudaMemsetAsync(e, 0x01, 4, w.stream));
    OVB_CUDA(cudaStreamSynchronize(w.stream));
  });
}

ordvec_status_t ovb_index_search_device(const ordvec_index_t* index, uint32_t method, const float* d_queries,
                                        uint64_t nq, uint64_t k, float* d_scores, int64_t* d_ids, void* stream) {
  return boundary([&] {
    const Index& ix = as_index(index);
    need_queries(d_queries, nq);
    const bool asym = method == OVB_SEARCH_ASYMMETRIC;
    if (method != OVB_SEARCH_DEFAULT && !asym) fail(ORDVEC_STATUS_BAD_ARGUMENT, "method must be 0 or 1");
    const bool rank_kind = ix.kind == ORDVEC_INDEX_KIND_RANK_QUANT || ix.kind == OVB_INDEX_KIND_RANK;
    if (!rank_kind && (asym || (ix.kind != ORDVEC_INDEX_KIND_BITMAP && ix.kind != OVB_INDEX_KIND_FASTSCAN)))
      fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "this index kind has no such full search");
    if (ix.kind == OVB_INDEX_KIND_RANK && ix.dim > kMaxDeviceRankDim)
      fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "device rank search supports dim <= 16384");
    if (ix.kind == ORDVEC_INDEX_KIND_RANK_QUANT && !asym && ix.dim > kMaxDeviceRankDim)
      fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "device rank transform supports dim <= 16384");
    const uint64_t ke = k < ix.n ? k : ix.n;
    if (!ke || !nq) return;
    if (!d_scores || !d_ids) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    Workspace& w = workspace();
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t got = 0;
    int mode = 0;
    switch (ix.kind) {
      case ORDVEC_INDEX_KIND_RANK_QUANT:
        got = asym ? engine_rankquant_full(ix, d_queries, nq, ke, w, st)
                   : engine_rankquant_symmetric(ix, d_queries, nq, ke, w, st);
        break;
      case OVB_INDEX_KIND_RANK:
        got = engine_rank_full(ix, d_queries, nq, ke, asym, w, st);
        break;
      case ORDVEC_INDEX_KIND_BITMAP:
        got = engine_bitmap_full(ix, d_queries, nq, ke, w, st);
        mode = 1;
        break;
      default:
        got = engine_fastscan_full(ix, d_queries, nq, ke, w, st);
    }
    launch_keys_to_results(w.out_keys.as<uint32_t>(), w.out_ids.as<uint32_t>(), nq * got, mode, ix.n_top, d_scores,
                           d_ids, st);
  });
}

ordvec_status_t ovb_two_stage_profile(const ordvec_index_t* rq, const ordvec_index_t* stage1,
                                      const float* d_queries, uint64_t nq, uint64_t m, uint64_t k,
                                      float* d_scores, int64_t* d_ids, void* stream, float* stage_ms) {
  return boundary([&] {
    const Index& r = as_index(rq);
    const Index& s = as_index(stage1);
    need_queries(d_queries, nq);
    if (!stage_ms) fail(ORDVEC_STATUS_NULL_POINTER, "stage_ms pointer is NULL");
    for (int i = 0; i < 6; i++) stage_ms[i] = 0.0f;
    if (!nq || !k || !r.n) return;
    if (!d_scores || !d_ids) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    Workspace& w = workspace();
    for (auto& e : w.prof_ev)
      if (!e) OVB_CUDA(cudaEventCreate(&e));
    cudaStream_t st = (cudaStream_t)stream;
    w.prof = true;
    try {
      uint32_t got = engine_two_stage(r, s, d_queries, nq, m, k, w, st);
      launch_keys_to_results(w.out_keys.as<uint32_t>(), w.out_ids.as<uint32_t>(), nq * got, 0, 0, d_scores, d_ids,
                             st);
    } catch (...) {
      w.prof = false;
      throw;
    }
    w.prof = false;
    OVB_CUDA(cudaStreamSynchronize(st));
    // event order: 0 start, 1 prep, 6 threshold, 2 scan, 3 select, 4 rerank, 5 final
    static const int order[7] = {0, 1, 6, 2, 3, 4, 5};
    for (int i = 0; i < 6; i++)
      OVB_CUDA(cudaEventElapsedTime(&stage_ms[i], w.prof_ev[order[i]], w.prof_ev[order[i + 1]]));
    OVB_CUDA(cudaStreamSynchronize(w.stream));
    check_tc(w);
  });
}

uint64_t ovb_last_launch_count(void) { return tl_last_launches; }

ordvec_status_t ovb_set_device(int device) {
  return boundary([&] {
    ensure_device();
    OVB_CUDA(cudaSetDevice(device));
  });
}

}  // extern "C"
