// Device pipelines: scan -> key matrix -> exact top-k select, and the fused
// two-stage (candidate generation -> asymmetric rerank) flow.
//
// Each pipeline takes device query rows and leaves its result in the calling
// thread's workspace (out_keys / out_ids, rows of k_eff entries, sentinel
// padded).  Queries are processed in chunks so the key matrix (nq_chunk x n
// u32) stays within a fixed HBM budget (OVB_KEYS_BUDGET_MB, default 2048).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "ovb_host.h"

namespace ovb {

namespace {

uint64_t keys_budget() {
  static const uint64_t b = [] {
    const char* e = getenv("OVB_KEYS_BUDGET_MB");
    uint64_t mb = e ? strtoull(e, nullptr, 10) : 2048;
    return (mb ? mb : 2048) << 20;
  }();
  return b;
}

// rankquant_norm (src/rank.rs:275-280) and 1/norm in f32, as the reference.
float rankquant_norm_f32(uint32_t dim, uint32_t bits) {
  const double n = (double)(1u << bits);
  return (float)std::sqrt((double)dim * ((n * n - 1.0) / 12.0));
}

float inv_rankquant_norm(uint32_t dim, uint32_t bits) { return 1.0f / rankquant_norm_f32(dim, bits); }

void select_rows(Workspace& w, const uint32_t* keys, const uint32_t* ids, const uint64_t* row_off,
                 uint64_t ld, uint64_t n, uint64_t rows, uint32_t k, uint32_t key_bits,
                 uint32_t id_bits, uint32_t* out_keys, uint32_t* out_ids, cudaStream_t st,
                 const uint32_t* row_len = nullptr, bool ordered = true) {
  SelectArgs a{keys, ids, row_off, ld, n, k, key_bits, id_bits, out_keys, out_ids, row_len, ordered ? 0u : 1u};
  size_t se = select_rows_scratch_elems(rows, k, row_off ? 0 : n);
  uint64_t* scratch = se ? (uint64_t*)w.scratch.ensure(se * 8) : nullptr;
  launch_select_rows(a, rows, scratch, st);
}

// scan(q0, qn, keys) writes keys[qn][n]; rows are selected into out[nq][k].
template <class F>
void full_scan_select(Workspace& w, uint64_t nq, uint64_t n, uint32_t k, uint32_t key_bits,
                      uint32_t* out_keys, uint32_t* out_ids, cudaStream_t st, F&& scan) {
  const uint64_t per_q = n * 4;
  uint64_t qc = keys_budget() / per_q;
  if (qc < 1) qc = 1;
  if (qc > nq) qc = nq;
  uint32_t* keys = (uint32_t*)w.keys.ensure(qc * per_q);
  const uint32_t id_bits = bits_for(n - 1);
  for (uint64_t q0 = 0; q0 < nq; q0 += qc) {
    const uint64_t qn = nq - q0 < qc ? nq - q0 : qc;
    scan(q0, qn, keys);
    w.mark(st, 2);
    select_rows(w, keys, nullptr, nullptr, n, n, qn, k, key_bits, id_bits, out_keys + q0 * k,
                out_ids + q0 * k, st, nullptr, !w.cand_unordered);
    w.mark(st, 3);
  }
}

float* normalised(Workspace& w, const float* d_q, uint64_t nq, uint32_t dim, cudaStream_t st) {
  float* qu = (float*)w.q_unit.ensure(nq * dim * 4);
  launch_l2_normalise(d_q, nq, dim, qu, st);
  return qu;
}

// Tensor-core FastScan for batches of at least 32 queries (one tile of the
// one-hot GEMM needs N >= 16 and pays off from ~32); OVB_FASTSCAN_TC=0/1 forces.
bool use_fastscan_tc(uint64_t nq) {
  const char* e = getenv("OVB_FASTSCAN_TC");
  if (e && e[0] == '0') return false;
  if (e && e[0] == '1') return true;
  return nq >= 32;
}

// Exact threshold filter for batched FastScan candidate generation (m << n).
//  1. score an evenly spread sample (every `stride`-th 32-doc block) and take,
//     per query, the r-th smallest sample key as the threshold thr;
//  2. rescore every doc, keeping only (key, doc) with key <= thr;
//  3. a query that kept c docs with m <= c <= cap kept every key <= its m-th
//     smallest key (at least m keys are <= thr), so the top-m of the kept set,
//     ties by doc id included, is the top-m of the whole index.  A chunk where
//     some query kept fewer than m or more than cap docs is redone through the
//     full key matrix.
// r is sized so a query keeps about `mult` * m docs (default 3): fewer than m
// would need the sample to over-represent the top-m ~3x, which for the default
// sample (>= 8192 docs) is a many-sigma event; the fallback keeps it exact.
struct FilterPlan {
  uint32_t stride;
  uint64_t n_s;
  uint32_t r;
  uint32_t cap;
};

bool filter_plan(uint64_t n, uint32_t m, FilterPlan& p) {
  const char* e = getenv("OVB_FASTSCAN_FILTER");
  if (e && e[0] == '0') return false;
  const bool force = e && e[0] == '1';
  if (!m || !n || (!force && (n < 32768 || (uint64_t)m * 32 > n))) return false;
  uint32_t stride = 1;
  // the sample pass costs about one CTA wave per 256 x 256 tile set, whatever
  // the doc count, so the sample is kept near 4-8K docs (one wave at <= 256
  // queries); the stride stops at 64, or at 128 from 4M docs (the sample's
  // dense keys and their select take a visible share of a batch there, and
  // the rank r of the threshold stays in the tens), and at 256 from 8M docs
  const uint32_t max_stride = n >= 8000000 ? 256 : n >= 4000000 ? 128 : 64;
  while (stride < max_stride && n / (2ull * stride) >= 4096) stride <<= 1;
  const uint64_t n_s = fastscan_tc_sample_docs(n, stride);
  const char* me = getenv("OVB_FASTSCAN_SAMPLE_MULT");
  const double mult = me ? strtod(me, nullptr) : 3.0;
  double rr = std::ceil(mult * (double)m * (double)n_s / (double)n) + (me ? 0.0 : 16.0);
  if (rr < 1.0) rr = 1.0;
  if (rr > (double)n_s) rr = (double)n_s;
  p.stride = stride;
  p.n_s = n_s;
  p.r = (uint32_t)rr;
  // A query keeps about r * stride docs (relative spread ~ 1 / sqrt(r)); the
  // capacity covers twice that as well as 8m, since one query over it sends
  // its whole chunk through the key matrix (with m = 320 at stride 128: r = 24,
  // ~3,100 kept, and 8m + 2048 alone overflowed for ~0.7 % of queries).
  const uint64_t by_m = 8ull * m + 2048, by_r = 2ull * p.r * stride + 4096;
  uint64_t cap = by_m > by_r ? by_m : by_r;
  if (cap > n + 32) cap = n + 32;
  p.cap = (uint32_t)((cap + 31) / 32 * 32);
  return true;
}

// Stage-1 top-m rows through the sampled threshold filter.
//   sample(q0, qn, keys)                 sample keys, rows of fp.n_s
//   filter(q0, qn, thr, pos, cnt, fk, fi) filtering scan; thr / pos: the r-th
//                                        sample key and its sample position,
//                                        row stride fp.r
//   dense(qa, qn)                        rows [qa, qa + qn) through the full key matrix
template <class Sample, class Filter, class Dense>
void filtered_select(Workspace& w, uint64_t n, uint64_t nq, uint32_t me, const FilterPlan& fp, uint32_t key_bits,
                     uint32_t* sk, uint32_t* si, cudaStream_t st, Sample&& sample, Filter&& filter,
                     Dense&& dense) {
  const uint64_t per_q = fp.n_s * 4 + (uint64_t)fp.r * 8 + (uint64_t)fp.cap * 8 + 4;
  uint64_t qc = keys_budget() / per_q;
  if (qc < 1) qc = 1;
  if (qc > nq) qc = nq;
  uint32_t* smp = (uint32_t*)w.smp_keys.ensure(qc * fp.n_s * 4);
  uint32_t* tk = (uint32_t*)w.thr_keys.ensure(qc * fp.r * 4);
  uint32_t* ti = (uint32_t*)w.thr_ids.ensure(qc * fp.r * 4);
  uint32_t* fk = (uint32_t*)w.f_keys.ensure(qc * fp.cap * 4);
  uint32_t* fi = (uint32_t*)w.f_ids.ensure(qc * fp.cap * 4);
  uint32_t* cnt = (uint32_t*)w.f_cnt.ensure(qc * 4);
  uint32_t* flag = (uint32_t*)w.f_flag.ensure(4);
  uint32_t* flag_h = (uint32_t*)w.f_flag_host.ensure(4);
  for (uint64_t q0 = 0; q0 < nq; q0 += qc) {
    const uint64_t qn = nq - q0 < qc ? nq - q0 : qc;
    sample(q0, qn, smp);
    select_rows(w, smp, nullptr, nullptr, fp.n_s, fp.n_s, qn, fp.r, key_bits, bits_for(fp.n_s - 1), tk, ti, st);
    w.mark(st, 6);
    OVB_CUDA(cudaMemsetAsync(cnt, 0, qn * 4, st));
    OVB_CUDA(cudaMemsetAsync(flag, 0, 4, st));
    filter(q0, qn, tk + (fp.r - 1), ti + (fp.r - 1), cnt, fk, fi);
    launch_filter_check(cnt, qn, me, fp.cap, flag, st);
    OVB_CUDA(cudaMemcpyAsync(flag_h, flag, 4, cudaMemcpyDeviceToHost, st));
    OVB_CUDA(cudaStreamSynchronize(st));
    if (*flag_h) {
      dense(q0, qn);
      continue;
    }
    w.mark(st, 2);
    select_rows(w, fk, fi, nullptr, fp.cap, fp.cap, qn, me, key_bits, bits_for(n - 1), sk + q0 * me, si + q0 * me,
                st, cnt, !w.cand_unordered);
    w.mark(st, 3);
  }
}

// Tensor-core overlap scan for sign bitmaps (Hamming), constant-weight bitmaps
// and identity-weight multi-bucket bitmaps: batches of at least 32 queries, and
// from 8 queries on indices of at least 2^20 rows whose top-m takes the
// sampled-threshold filter (the CUDA-core form would write nq key rows of n
// keys and select m from each: milliseconds at millions of rows, where the
// filtered scan costs about the same for 8 queries as for 256);
// OVB_BITMAP_TC=0/1 forces.
bool use_bitmap_tc(uint64_t nq, uint64_t n, uint32_t m) {
  const char* e = getenv("OVB_BITMAP_TC");
  if (e && e[0] == '0') return false;
  if (e && e[0] == '1') return true;
  FilterPlan fp;
  return nq >= 32 || (nq >= 8 && n >= (1ull << 20) && filter_plan(n, m, fp));
}

// Stage-1 top-m of a bitmap-family index on the tensor cores: key_kind 0 for a
// constant-weight bitmap, 1 for a multi-bucket bitmap with identity weights,
// 2 for a sign bitmap (Hamming); qb = query words (qpv per query).
void bitmap_tc_candidates(const Index& s1, const uint64_t* qb, uint32_t qpv, uint32_t key_kind, uint32_t key_bits,
                          uint64_t nq, uint32_t me, uint32_t* sk, uint32_t* si, Workspace& w, cudaStream_t st) {
  const uint64_t n = s1.n;
  const uint64_t row = (uint64_t)bitmap_tc_kblocks(qpv) * 128;
  uint8_t* qx = (uint8_t*)w.lut.ensure(nq * row);
  uint32_t* qpop = key_kind == 2 ? (uint32_t*)w.bias.ensure(nq * 4) : nullptr;  // bias is FastScan's
  launch_bitmap_tc_query(qb, nq, qpv, qx, qpop, st);
  const uint64_t* words = s1.codes.as<uint64_t>();
  // the filter's query operand on the FP4 tensor cores, built with the int8 one
  // (the sample scan writes every key and stays on int8)
  const uint64_t row4 = (uint64_t)bitmap_fp4_kblocks(qpv) * 128;
  uint8_t* q4 = nullptr;
  uint32_t* err = w.tc_err_word(st);
  auto dense = [&](uint64_t qa, uint64_t qn) {
    full_scan_select(w, qn, n, me, key_bits, sk + qa * me, si + qa * me, st,
                     [&](uint64_t q0, uint64_t qm, uint32_t* keys) {
                       launch_bitmap_scan_tc(words, n, qpv, key_kind, s1.n_top, qpop ? qpop + qa + q0 : nullptr,
                                             qx + (qa + q0) * row, qm, 1, keys, n, err, st);
                     });
  };
  FilterPlan fp;
  if (!filter_plan(n, me, fp)) {
    w.mark(st, 6);  // no sampling stage
    dense(0, nq);
    return;
  }
  if (bitmap_fp4_usable(qpv)) {
    q4 = (uint8_t*)w.q_nib.ensure(nq * row4);
    launch_bitmap_fp4_query(qb, nq, qpv, q4, st);
  }
  filtered_select(
      w, n, nq, me, fp, key_bits, sk, si, st,
      [&](uint64_t q0, uint64_t qn, uint32_t* smp) {
        launch_bitmap_scan_tc(words, n, qpv, key_kind, s1.n_top, qpop ? qpop + q0 : nullptr, qx + q0 * row, qn,
                              fp.stride, smp, fp.n_s, err, st);
      },
      [&](uint64_t q0, uint64_t qn, const uint32_t* thr, const uint32_t* pos, uint32_t* cnt, uint32_t* fk,
          uint32_t* fi) {
        launch_bitmap_filter_tc(words, n, qpv, key_kind, s1.n_top, qpop ? qpop + q0 : nullptr, qx + q0 * row,
                                q4 ? q4 + q0 * row4 : nullptr, qn, thr, pos, fp.stride, fp.r, cnt, fp.cap, fk, fi, err,
                                st);
      },
      dense);
}

void require_kind(const Index& ix, uint32_t kind, const char* what) {
  if (ix.kind != kind) fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, std::string(what) + ": wrong index kind");
}

}  // namespace

uint64_t engine_keys_budget() { return keys_budget(); }

uint64_t engine_stage1_bytes(const Index& s1, uint64_t nq, uint64_t m) {
  const uint64_t n = s1.n;
  const uint32_t me = (uint32_t)(m < n ? m : n);
  const bool bitmap = s1.kind == OVB_INDEX_KIND_SIGN_BITMAP || s1.kind == ORDVEC_INDEX_KIND_BITMAP;
  FilterPlan fp;
  if (bitmap && me && use_bitmap_tc(nq, n, me) && filter_plan(n, me, fp))
    return nq * (fp.n_s * 4 + (uint64_t)fp.r * 8 + (uint64_t)fp.cap * 8 + 4);
  const uint64_t keys = nq * n * 4;
  return keys < keys_budget() ? keys : keys_budget();
}

uint64_t default_candidate_count(uint64_t k, uint64_t space) {
  // TwoStageCandidatePolicy::default() (src/quant.rs:242-262): min 256, k*32.
  if (k == 0 || space == 0) return 0;
  uint64_t prod = k > UINT64_MAX / 32 ? UINT64_MAX : k * 32;
  uint64_t c = prod > 256 ? prod : 256;
  return c < space ? c : space;
}

// Batched full scans use the split-BF16 tensor-core scan (with the exact FP64
// rescoring below) from 64 queries on eligible shapes; OVB_RANK_TC=0/1 forces.
bool use_rank_tc(const Index& rq, uint64_t nq) {
  const char* e = getenv("OVB_RANK_TC");
  if (!rank_tc_eligible(rq.dim, rq.bits)) return false;
  if (e && e[0] == '0') return false;
  if (e && e[0] == '1') return true;
  return nq >= 64 && rq.n >= 4096;
}

// Split-BF16 filter for rows of kp candidates: the sample-threshold plan with
// kp in place of m (OVB_SPLIT_FILTER=0 disables).
static bool split_filter_plan(uint64_t n, uint64_t kp, FilterPlan& fp) {
  const char* e = getenv("OVB_SPLIT_FILTER");
  if (e && e[0] == '0') return false;
  return kp <= kSelectSmemCap && filter_plan(n, (uint32_t)kp, fp);
}

static uint64_t split_filter_bytes_per_query(const FilterPlan& fp, uint64_t kp) {
  return fp.n_s * 4 + (uint64_t)fp.r * 8 + (uint64_t)fp.cap * 8 + 4 + kp * 12 + 8;
}

// Enqueues the filtered split-BF16 pipeline for qn queries (no host
// synchronisation, graph-capturable): sample scan, each query's r-th sample
// key as threshold, filtered scan, top-kp of the kept docs by split score,
// margin test, FP64 rescoring of the kp, top-ke into out_keys / out_ids.
// *d_flag |= 1 when some query kept fewer than kp or more than cap docs, or
// its kp-th split score is within twice the error bound of its k-th: the
// result is then not known to be exact and the caller redoes the rows.
// Kept sets are prefixes of the split-key order, so their top-kp is the
// whole index's.
static void split_filtered(const Index& rq, const uint16_t* qs, const float* qu, const float* l1, float inv_norm,
                           uint64_t qn, uint32_t ke, uint32_t kp, const FilterPlan& fp, uint32_t q_per_tile,
                           uint32_t* d_flag, uint32_t* out_keys, uint32_t* out_ids, Workspace& w, cudaStream_t st) {
  const uint64_t n = rq.n;
  const uint32_t dim = rq.dim, bits = rq.bits, id_bits = bits_for(n - 1);
  const uint8_t* codes = rq.codes.as<uint8_t>();
  uint32_t* err = w.tc_err_word(st);
  uint32_t* smp = (uint32_t*)w.smp_keys.ensure(qn * fp.n_s * 4);
  launch_rank_scan_tc(codes, n, dim, bits, qs, qn, inv_norm, fp.stride, smp, fp.n_s, q_per_tile, err, st);
  uint32_t* tk = (uint32_t*)w.thr_keys.ensure(qn * fp.r * 4);
  uint32_t* ti = (uint32_t*)w.thr_ids.ensure(qn * fp.r * 4);
  select_rows(w, smp, nullptr, nullptr, fp.n_s, fp.n_s, qn, fp.r, 32, bits_for(fp.n_s - 1), tk, ti, st);
  w.mark(st, 6);
  uint32_t* cnt = (uint32_t*)w.f_cnt.ensure(qn * 4);
  uint32_t* fk = (uint32_t*)w.f_keys.ensure(qn * fp.cap * 4);
  uint32_t* fi = (uint32_t*)w.f_ids.ensure(qn * fp.cap * 4);
  OVB_CUDA(cudaMemsetAsync(cnt, 0, qn * 4, st));
  launch_rank_filter_tc(codes, n, dim, bits, qs, qn, inv_norm, tk + (fp.r - 1), fp.r, cnt, fp.cap, fk, fi, q_per_tile,
                        err, st);
  launch_filter_check(cnt, qn, kp, fp.cap, d_flag, st);
  w.mark(st, 2);
  uint32_t* ck = (uint32_t*)w.sel_keys.ensure(qn * kp * 4);
  uint32_t* ci = (uint32_t*)w.sel_ids.ensure(qn * kp * 4);
  select_rows(w, fk, fi, nullptr, fp.cap, fp.cap, qn, kp, 32, id_bits, ck, ci, st, cnt);
  launch_clamp_ids(ci, qn * kp, (uint32_t)n, st);  // a row that kept < kp docs ends in sentinels
  launch_split_margin(ck, qn, kp, ke, l1, split_error_bound(dim, bits, inv_norm), d_flag, st);
  w.mark(st, 3);
  uint64_t* off = (uint64_t*)w.off.ensure((qn + 1) * 8);
  launch_uniform_offsets(off, qn, kp, st);
  uint32_t* k2 = (uint32_t*)w.keys2.ensure(qn * kp * 4);
  launch_asym_subset(codes, dim, bits, qu, qn, off, ci, kp, inv_norm, k2, st);
  w.mark(st, 4);
  select_rows(w, k2, ci, off, 0, 0, qn, ke, 32, id_bits, out_keys, out_ids, st);
  w.mark(st, 5);
}

// Split-BF16 search of prepared query rows qu (nq x dim f32) scored as
// sum_j qu[j] (code_j - c) * inv_norm: the unit query and 1/norm for
// search_asymmetric, the centred query buckets and 1/norm^2 for the symmetric
// search.  The error bound is linear in |qu|_1 and inv_norm, so both share it.
static uint32_t split_search(const Index& rq, const float* qu, float inv_norm, uint64_t nq, uint64_t k, bool exact,
                             Workspace& w, cudaStream_t st, uint32_t q_per_tile) {
  if (!rank_tc_eligible(rq.dim, rq.bits))
    fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "split-BF16 scan needs dim to be a multiple of 64");
  const uint64_t n = rq.n;
  const uint32_t ke = (uint32_t)(k < n ? k : n);
  if (!ke || !nq) return ke;
  const uint32_t dim = rq.dim, bits = rq.bits;
  const float bound = split_error_bound(dim, bits, inv_norm);
  uint16_t* qs = (uint16_t*)w.q_split.ensure(nq * 2 * dim * 2);
  float* l1 = (float*)w.q_l1.ensure(nq * 4);
  launch_split_queries(qu, nq, dim, qs, l1, st);
  uint32_t* ok = (uint32_t*)w.out_keys.ensure(nq * ke * 4);
  uint32_t* oi = (uint32_t*)w.out_ids.ensure(nq * ke * 4);
  uint32_t* flag = (uint32_t*)w.f_flag.ensure(4);
  uint32_t* flag_h = (uint32_t*)w.f_flag_host.ensure(4);
  const uint32_t id_bits = bits_for(n - 1);
  w.split_kp = 0;
  const uint64_t kp0 = std::min<uint64_t>(std::max<uint64_t>(2ull * ke, ke + 64ull), n);
  FilterPlan fp;
  // rows that passed the filtered pipeline; the others take the key matrix below
  std::vector<char> done;
  if (exact && split_filter_plan(n, kp0, fp)) {
    uint64_t fc = keys_budget() / split_filter_bytes_per_query(fp, kp0);
    if (fc < 1) fc = 1;
    done.assign(nq, 0);
    for (uint64_t q0 = 0; q0 < nq; q0 += fc) {
      const uint64_t qn = nq - q0 < fc ? nq - q0 : fc;
      OVB_CUDA(cudaMemsetAsync(flag, 0, 4, st));
      split_filtered(rq, qs + q0 * 2 * dim, qu + q0 * dim, l1 + q0, inv_norm, qn, ke, (uint32_t)kp0, fp, q_per_tile,
                     flag, ok + q0 * ke, oi + q0 * ke, w, st);
      OVB_CUDA(cudaMemcpyAsync(flag_h, flag, 4, cudaMemcpyDeviceToHost, st));
      OVB_CUDA(cudaStreamSynchronize(st));
      if (!*flag_h) {
        std::fill(done.begin() + q0, done.begin() + q0 + qn, 1);
        w.split_kp = std::max<uint64_t>(w.split_kp, kp0);
      }
    }
  }
  uint64_t qc = keys_budget() / (n * 4);
  if (qc < 1) qc = 1;
  if (qc > nq) qc = nq;
  uint32_t* keys = nullptr;
  for (uint64_t q0 = 0; q0 < nq; q0 += qc) {
    const uint64_t qn = nq - q0 < qc ? nq - q0 : qc;
    if (!done.empty() && std::all_of(done.begin() + q0, done.begin() + q0 + qn, [](char c) { return c != 0; }))
      continue;
    if (!keys) keys = (uint32_t*)w.keys.ensure(qc * n * 4);
    launch_rank_scan_tc(rq.codes.as<uint8_t>(), n, dim, bits, qs + q0 * 2 * dim, qn, inv_norm, 1, keys, n,
                        q_per_tile, w.tc_err_word(st), st);
    w.mark(st, 2);
    if (!exact) {
      select_rows(w, keys, nullptr, nullptr, n, n, qn, ke, 32, id_bits, ok + q0 * ke, oi + q0 * ke, st);
      w.mark(st, 3);
      continue;
    }
    // candidates: the top kp by split score, kp grown until the kp-th is more
    // than twice the bound below the k-th, so every doc whose exact score can
    // reach the exact top-k is a candidate; the key matrix is reused
    uint64_t kp = std::max<uint64_t>(2ull * ke, ke + 64ull);
    for (;;) {
      if (kp > n) kp = n;
      uint32_t* tk = (uint32_t*)w.thr_keys.ensure(qn * kp * 4);
      uint32_t* ti = (uint32_t*)w.thr_ids.ensure(qn * kp * 4);
      select_rows(w, keys, nullptr, nullptr, n, n, qn, (uint32_t)kp, 32, id_bits, tk, ti, st);
      if (kp == n) break;
      OVB_CUDA(cudaMemsetAsync(flag, 0, 4, st));
      launch_split_margin(tk, qn, (uint32_t)kp, ke, l1 + q0, bound, flag, st);
      OVB_CUDA(cudaMemcpyAsync(flag_h, flag, 4, cudaMemcpyDeviceToHost, st));
      OVB_CUDA(cudaStreamSynchronize(st));
      if (!*flag_h) break;
      kp *= 4;
    }
    w.split_kp = std::max<uint64_t>(w.split_kp, kp);
    uint64_t* off = (uint64_t*)w.off.ensure((qn + 1) * 8);
    launch_uniform_offsets(off, qn, (uint32_t)kp, st);
    uint32_t* k2 = (uint32_t*)w.keys2.ensure(qn * kp * 4);
    const uint32_t* ti = w.thr_ids.as<uint32_t>();
    launch_asym_subset(rq.codes.as<uint8_t>(), dim, bits, qu + q0 * dim, qn, off, ti, kp, inv_norm, k2, st);
    select_rows(w, k2, ti, off, 0, 0, qn, ke, 32, id_bits, ok + q0 * ke, oi + q0 * ke, st);
    w.mark(st, 3);
  }
  return ke;
}

uint32_t engine_rankquant_full_split(const Index& rq, const float* d_q, uint64_t nq, uint64_t k, bool exact,
                                     Workspace& w, cudaStream_t st, uint32_t q_per_tile) {
  require_kind(rq, ORDVEC_INDEX_KIND_RANK_QUANT, "search_asymmetric");
  if (!rank_tc_eligible(rq.dim, rq.bits))
    fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "split-BF16 scan needs dim to be a multiple of 64");
  const uint64_t ke = k < rq.n ? k : rq.n;
  if (!ke || !nq) return (uint32_t)ke;
  const float* qu = normalised(w, d_q, nq, rq.dim, st);
  return split_search(rq, qu, inv_rankquant_norm(rq.dim, rq.bits), nq, k, exact, w, st, q_per_tile);
}

bool split_fixed_fits(const Index& rq, uint64_t nq, uint64_t k) {
  const uint64_t n = rq.n, ke = k < n ? k : n;
  const uint64_t kp = std::min<uint64_t>(std::max<uint64_t>(2 * ke, ke + 64), n);
  FilterPlan fp;
  if (split_filter_plan(n, kp, fp) && nq * split_filter_bytes_per_query(fp, kp) <= keys_budget()) return true;
  return nq * n * 4 <= keys_budget();
}

uint32_t engine_rankquant_split_fixed(const Index& rq, const float* d_q, uint64_t nq, uint64_t k, uint64_t kp,
                                      uint32_t q_per_tile, uint32_t* d_flag, Workspace& w, cudaStream_t st) {
  require_kind(rq, ORDVEC_INDEX_KIND_RANK_QUANT, "search_asymmetric");
  const uint64_t n = rq.n;
  const uint32_t ke = (uint32_t)(k < n ? k : n);
  if (!ke || !nq) return ke;
  if (kp > n) kp = n;
  if (kp < ke) kp = ke;
  FilterPlan fp;
  const bool filtered = split_filter_plan(n, kp, fp) && nq * split_filter_bytes_per_query(fp, kp) <= keys_budget();
  if (!rank_tc_eligible(rq.dim, rq.bits) || (!filtered && nq * n * 4 > keys_budget()))
    fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "fixed split search: shape outside the single-chunk form");
  const uint32_t dim = rq.dim, bits = rq.bits, id_bits = bits_for(n - 1);
  const float* qu = normalised(w, d_q, nq, dim, st);
  const float inv_norm = inv_rankquant_norm(dim, bits);
  uint16_t* qs = (uint16_t*)w.q_split.ensure(nq * 2 * dim * 2);
  float* l1 = (float*)w.q_l1.ensure(nq * 4);
  launch_split_queries(qu, nq, dim, qs, l1, st);
  uint32_t* ok = (uint32_t*)w.out_keys.ensure(nq * ke * 4);
  uint32_t* oi = (uint32_t*)w.out_ids.ensure(nq * ke * 4);
  if (filtered) {
    split_filtered(rq, qs, qu, l1, inv_norm, nq, ke, (uint32_t)kp, fp, q_per_tile, d_flag, ok, oi, w, st);
    return ke;
  }
  uint32_t* keys = (uint32_t*)w.keys.ensure(nq * n * 4);
  launch_rank_scan_tc(rq.codes.as<uint8_t>(), n, dim, bits, qs, nq, inv_norm, 1, keys, n, q_per_tile,
                      w.tc_err_word(st), st);
  uint32_t* tk = (uint32_t*)w.thr_keys.ensure(nq * kp * 4);
  uint32_t* ti = (uint32_t*)w.thr_ids.ensure(nq * kp * 4);
  select_rows(w, keys, nullptr, nullptr, n, n, nq, (uint32_t)kp, 32, id_bits, tk, ti, st);
  if (kp < n) launch_split_margin(tk, nq, (uint32_t)kp, ke, l1, split_error_bound(dim, bits, inv_norm), d_flag, st);
  uint64_t* off = (uint64_t*)w.off.ensure((nq + 1) * 8);
  launch_uniform_offsets(off, nq, (uint32_t)kp, st);
  uint32_t* k2 = (uint32_t*)w.keys2.ensure(nq * kp * 4);
  launch_asym_subset(rq.codes.as<uint8_t>(), dim, bits, qu, nq, off, ti, kp, inv_norm, k2, st);
  select_rows(w, k2, ti, off, 0, 0, nq, ke, 32, id_bits, ok, oi, st);
  return ke;
}

uint32_t engine_rankquant_full(const Index& rq, const float* d_q, uint64_t nq, uint64_t k,
                               Workspace& w, cudaStream_t st) {
  require_kind(rq, ORDVEC_INDEX_KIND_RANK_QUANT, "search_asymmetric");
  if (use_rank_tc(rq, nq)) return engine_rankquant_full_split(rq, d_q, nq, k, true, w, st);
  const uint32_t ke = (uint32_t)(k < rq.n ? k : rq.n);
  if (!ke || !nq) return ke;
  const float* qu = normalised(w, d_q, nq, rq.dim, st);
  const float inv_norm = inv_rankquant_norm(rq.dim, rq.bits);
  uint32_t* ok = (uint32_t*)w.out_keys.ensure(nq * ke * 4);
  uint32_t* oi = (uint32_t*)w.out_ids.ensure(nq * ke * 4);
  full_scan_select(w, nq, rq.n, ke, 32, ok, oi, st, [&](uint64_t q0, uint64_t qn, uint32_t* keys) {
    launch_asym_scan(rq.codes.as<uint8_t>(), rq.n, rq.dim, rq.bits, qu + q0 * rq.dim, qn, inv_norm, keys,
                     rq.n, st);
  });
  return ke;
}

// RankQuant::search (src/quant.rs:629-695).  Query side of the LUT =
// bucket_centre(bucket(rank)), a half-integer; each LUT entry is a multiple of
// 1/4 and for b <= 4 every partial sum stays below 2^22 quarters, so the
// reference's sequential f32 sum is exact and equals the asymmetric scan's
// FP64 dot; (float)(dot * (double)inv_norm_sq) is then the reference's single
// f32 rounding of acc * inv_norm_sq (a product of two f32 is exact in f64).
uint32_t engine_rankquant_symmetric(const Index& rq, const float* d_q, uint64_t nq, uint64_t k, Workspace& w,
                                    cudaStream_t st) {
  require_kind(rq, ORDVEC_INDEX_KIND_RANK_QUANT, "search");
  const uint32_t ke = (uint32_t)(k < rq.n ? k : rq.n);
  if (!ke || !nq) return ke;
  float* qc = (float*)w.q_unit.ensure(nq * rq.dim * 4);
  launch_encode(6, d_q, nq, rq.dim, rq.bits, 0, 0, qc, 0, st);
  const float norm = rankquant_norm_f32(rq.dim, rq.bits);
  const float inv_norm_sq = 1.0f / (norm * norm);
  // batches: split-BF16 candidates (the centred buckets are exact in BF16, so
  // lo = 0) rescored exactly
  if (use_rank_tc(rq, nq)) return split_search(rq, qc, inv_norm_sq, nq, k, true, w, st, 0);
  uint32_t* ok = (uint32_t*)w.out_keys.ensure(nq * ke * 4);
  uint32_t* oi = (uint32_t*)w.out_ids.ensure(nq * ke * 4);
  full_scan_select(w, nq, rq.n, ke, 32, ok, oi, st, [&](uint64_t q0, uint64_t qn, uint32_t* keys) {
    launch_asym_scan(rq.codes.as<uint8_t>(), rq.n, rq.dim, rq.bits, qc + q0 * rq.dim, qn, inv_norm_sq, keys, rq.n,
                     st);
  });
  return ke;
}

// Rank::search / Rank::search_asymmetric (src/rank.rs:364-482).
uint32_t engine_rank_full(const Index& rk, const float* d_q, uint64_t nq, uint64_t k, bool asymmetric, Workspace& w,
                          cudaStream_t st) {
  require_kind(rk, OVB_INDEX_KIND_RANK, asymmetric ? "search_asymmetric" : "search");
  const uint32_t ke = (uint32_t)(k < rk.n ? k : rk.n);
  if (!ke || !nq) return ke;
  const uint16_t* ranks = rk.codes.as<uint16_t>();
  const uint32_t dim = rk.dim;
  uint32_t* ok = (uint32_t*)w.out_keys.ensure(nq * ke * 4);
  uint32_t* oi = (uint32_t*)w.out_ids.ensure(nq * ke * 4);
  if (asymmetric) {
    const float* qu = normalised(w, d_q, nq, dim, st);
    float* qsum = (float*)w.invq.ensure(nq * 4);
    full_scan_select(w, nq, rk.n, ke, 32, ok, oi, st, [&](uint64_t q0, uint64_t qn, uint32_t* keys) {
      launch_rank_asym_scan(ranks, rk.n, dim, qu + q0 * dim, qsum + q0, qn, keys, rk.n, st);
    });
  } else {
    uint16_t* qr = (uint16_t*)w.qbits.ensure(nq * dim * 2);
    launch_encode(5, d_q, nq, dim, 0, 0, 0, qr, 0, st);
    full_scan_select(w, nq, rk.n, ke, 32, ok, oi, st, [&](uint64_t q0, uint64_t qn, uint32_t* keys) {
      launch_rank_sym_scan(ranks, rk.n, dim, qr + q0 * dim, qn, keys, rk.n, st);
    });
  }
  return ke;
}

uint32_t engine_rankquant_subset(const Index& rq, const float* d_q, uint64_t nq,
                                 const uint64_t* d_off, const uint32_t* d_cands, uint64_t max_row,
                                 uint64_t k, Workspace& w, cudaStream_t st) {
  require_kind(rq, ORDVEC_INDEX_KIND_RANK_QUANT, "search_asymmetric_subset");
  const uint32_t ke = (uint32_t)(k < rq.n ? k : rq.n);
  if (!ke || !nq) return ke;
  const float* qu = normalised(w, d_q, nq, rq.dim, st);
  const float inv_norm = inv_rankquant_norm(rq.dim, rq.bits);
  // total entries = d_off[nq]; the caller sized keys2 through max_row * nq
  uint32_t* keys = (uint32_t*)w.keys2.ensure((max_row ? max_row : 1) * nq * 4);
  launch_asym_subset(rq.codes.as<uint8_t>(), rq.dim, rq.bits, qu, nq, d_off, d_cands, max_row, inv_norm,
                     keys, st);
  uint32_t* ok = (uint32_t*)w.out_keys.ensure(nq * ke * 4);
  uint32_t* oi = (uint32_t*)w.out_ids.ensure(nq * ke * 4);
  select_rows(w, keys, d_cands, d_off, 0, 0, nq, ke, 32, bits_for(rq.n - 1), ok, oi, st);
  return ke;
}

// Stage-1 candidates into w.sel_keys / w.sel_ids, rows of m_eff ids.
uint32_t engine_candidates(const Index& s1, const float* d_q, uint64_t nq, uint64_t m,
                           const float* d_weights, Workspace& w, cudaStream_t st, const float* q_unit) {
  const uint32_t me = (uint32_t)(m < s1.n ? m : s1.n);
  if (!me || !nq) return me;
  uint32_t* sk = (uint32_t*)w.sel_keys.ensure(nq * me * 4);
  uint32_t* si = (uint32_t*)w.sel_ids.ensure(nq * me * 4);
  const uint64_t n = s1.n;
  switch (s1.kind) {
    case OVB_INDEX_KIND_SIGN_BITMAP:
    case ORDVEC_INDEX_KIND_BITMAP: {
      const int mode = s1.kind == OVB_INDEX_KIND_SIGN_BITMAP ? 0 : 1;
      uint64_t* qb = (uint64_t*)w.qbits.ensure(nq * s1.qpv() * 8);
      if (mode == 0)
        launch_sign_query(d_q, nq, s1.dim, qb, st);
      else
        launch_bitmap_query(d_q, nq, s1.dim, s1.n_top, qb, st);
      w.mark(st, 1);
      const uint32_t key_bits = bits_for(mode == 0 ? s1.dim : s1.n_top);
      if (use_bitmap_tc(nq, n, me)) {  // sign: Hamming (key kind 2); bitmap: n_top - overlap (0)
        bitmap_tc_candidates(s1, qb, s1.qpv(), mode == 0 ? 2 : 0, key_bits, nq, me, sk, si, w, st);
        break;
      }
      w.mark(st, 6);  // no sampling stage
      full_scan_select(w, nq, n, me, key_bits, sk, si, st, [&](uint64_t q0, uint64_t qn, uint32_t* keys) {
        launch_popc_scan(mode, s1.codes.as<uint64_t>(), n, s1.qpv(), qb + q0 * s1.qpv(), qn, s1.n_top, keys,
                         n, st);
      });
      break;
    }
    case OVB_INDEX_KIND_FASTSCAN: {
      const float* qu = q_unit ? q_unit : normalised(w, d_q, nq, s1.dim, st);
      uint8_t* lut = (uint8_t*)w.lut.ensure(nq * s1.pairs_pad * 16);
      float* bias = (float*)w.bias.ensure(nq * 4);
      float* invq = (float*)w.invq.ensure(nq * 4);
      launch_fastscan_lut(qu, nq, s1.dim, s1.pairs_pad, lut, bias, invq, st);
      w.mark(st, 1);
      const float inv_norm = inv_rankquant_norm(s1.dim, 2);
      const uint8_t* codes = s1.codes.as<uint8_t>();
      const uint64_t lut_row = (uint64_t)s1.pairs_pad * 16;
      // rows [qa, qa + qn) through the full key matrix
      auto dense_rows = [&](uint64_t qa, uint64_t qn) {
        full_scan_select(w, qn, n, me, 32, sk + qa * me, si + qa * me, st,
                         [&](uint64_t q0, uint64_t qm, uint32_t* keys) {
                           const uint64_t qg = qa + q0;
                           if (use_fastscan_tc(qm))
                             launch_fastscan_scan_tc(codes, n, s1.pairs_pad, lut + qg * lut_row, bias + qg,
                                                     invq + qg, inv_norm, qm, 1, keys, n, w.tc_err_word(st), st);
                           else
                             launch_fastscan_scan(codes, n, s1.pairs_pad, lut + qg * lut_row, bias + qg, invq + qg,
                                                  inv_norm, qm, keys, n, st);
                         });
      };
      FilterPlan fp;
      if (!use_fastscan_tc(nq) || !filter_plan(n, me, fp)) {
        w.mark(st, 6);  // no sampling stage
        dense_rows(0, nq);
        break;
      }
      uint32_t* err = w.tc_err_word(st);
      filtered_select(
          w, n, nq, me, fp, 32, sk, si, st,
          [&](uint64_t q0, uint64_t qn, uint32_t* smp) {
            launch_fastscan_scan_tc(codes, n, s1.pairs_pad, lut + q0 * lut_row, bias + q0, invq + q0, inv_norm, qn,
                                    fp.stride, smp, fp.n_s, err, st);
          },
          [&](uint64_t q0, uint64_t qn, const uint32_t* thr, const uint32_t*, uint32_t* cnt, uint32_t* fk,
              uint32_t* fi) {
            launch_fastscan_filter_tc(codes, n, s1.pairs_pad, lut + q0 * lut_row, bias + q0, invq + q0, inv_norm,
                                      qn, thr, fp.r, cnt, fp.cap, fk, fi, (uint64_t)fp.r * n / fp.n_s, err, st);
          },
          dense_rows);
      break;
    }
    case OVB_INDEX_KIND_MULTIBUCKET: {
      const uint32_t nb = s1.nb(), qpb = s1.dim / 64;
      uint64_t* qb = (uint64_t*)w.qbits.ensure(nq * nb * qpb * 8);
      launch_multibucket_query(d_q, nq, s1.dim, s1.bits, qb, st);
      w.mark(st, 1);
      if (!d_weights && use_bitmap_tc(nq, n, me)) {
        // identity weights: the f32 sum over (a, a) of popcount(Q_a AND D_a)
        // is the integer overlap of the concatenated bucket rows (exact below 2^24)
        bitmap_tc_candidates(s1, qb, nb * qpb, 1, 32, nq, me, sk, si, w, st);
        break;
      }
      w.mark(st, 6);  // no sampling stage
      const float* wts = d_weights;
      if (!wts) {  // diagonal weights (src/multi_bucket.rs:157-164)
        std::vector<float> diag(nb * nb, 0.0f);
        for (uint32_t a = 0; a < nb; a++) diag[a * nb + a] = 1.0f;
        float* dw = (float*)w.weights.ensure(nb * nb * 4);
        OVB_CUDA(cudaMemcpyAsync(dw, diag.data(), nb * nb * 4, cudaMemcpyHostToDevice, st));
        OVB_CUDA(cudaStreamSynchronize(st));
        wts = dw;
      }
      full_scan_select(w, nq, n, me, 32, sk, si, st, [&](uint64_t q0, uint64_t qn, uint32_t* keys) {
        launch_multibucket_scan(s1.codes.as<uint64_t>(), n, qpb, nb, qb + q0 * nb * qpb, wts, qn, keys, n, st);
      });
      break;
    }
    default:
      fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "index kind cannot generate candidates");
  }
  return me;
}

uint32_t engine_bitmap_full(const Index& bm, const float* d_q, uint64_t nq, uint64_t k,
                            Workspace& w, cudaStream_t st) {
  require_kind(bm, ORDVEC_INDEX_KIND_BITMAP, "Bitmap::search");
  const uint32_t ke = engine_candidates(bm, d_q, nq, k, nullptr, w, st);
  if (ke && nq) {
    OVB_CUDA(cudaMemcpyAsync(w.out_keys.ensure(nq * ke * 4), w.sel_keys.p, nq * ke * 4,
                             cudaMemcpyDeviceToDevice, st));
    OVB_CUDA(cudaMemcpyAsync(w.out_ids.ensure(nq * ke * 4), w.sel_ids.p, nq * ke * 4,
                             cudaMemcpyDeviceToDevice, st));
  }
  return ke;
}

uint32_t engine_fastscan_full(const Index& fs, const float* d_q, uint64_t nq, uint64_t k,
                              Workspace& w, cudaStream_t st) {
  require_kind(fs, OVB_INDEX_KIND_FASTSCAN, "RankQuantFastscan::search");
  const uint32_t ke = engine_candidates(fs, d_q, nq, k, nullptr, w, st);
  if (ke && nq) {
    OVB_CUDA(cudaMemcpyAsync(w.out_keys.ensure(nq * ke * 4), w.sel_keys.p, nq * ke * 4,
                             cudaMemcpyDeviceToDevice, st));
    OVB_CUDA(cudaMemcpyAsync(w.out_ids.ensure(nq * ke * 4), w.sel_ids.p, nq * ke * 4,
                             cudaMemcpyDeviceToDevice, st));
  }
  return ke;
}

// How a two-stage search reranks its uniform candidate rows (me per query,
// top-ke): the caller's OVB_RERANK_* mode; OVB_RERANK_AUTO takes the FP64
// per-query tables, measured faster than the exact split-BF16 form at the
// benchmark shapes (N=10M dim 768 b=2, 1,024 x 2,000 candidates: 0.38 vs
// 0.61 ms; N=171,332 dim 1024: 0.23 vs 0.36 ms), unless OVB_RERANK_TC=1 asks
// for the split-BF16 tensor-core rerank (eligible shapes, >= 16 queries, rows
// long enough for the rescoring set kp to be a real subset).
static uint32_t rerank_mode(const Workspace& w, const Index& rq, uint64_t nq, uint32_t me, uint32_t ke) {
  if (w.rerank_mode == OVB_RERANK_SPLIT_RAW) return rerank_tc_eligible(rq.dim, rq.bits) ? w.rerank_mode : OVB_RERANK_FP64;
  if (w.rerank_mode != OVB_RERANK_AUTO) return w.rerank_mode;
  if (!rerank_tc_eligible(rq.dim, rq.bits)) return OVB_RERANK_FP64;
  const char* e = getenv("OVB_RERANK_TC");
  if (!(e && e[0] == '1')) return OVB_RERANK_FP64;
  return nq >= 16 && (uint64_t)me >= 4ull * ke + 64 ? OVB_RERANK_SPLIT : OVB_RERANK_FP64;
}

// Split-BF16 rerank of the uniform candidate rows in w.sel_ids (me per query):
// split queries, the tensor-core rerank (keys2), then either the raw top-ke of
// the split scores (raw) or the exact form -- the top-kp by split score with
// kp = min(me, 2 ke + 32), the margin test (the kp-th split score more than
// twice the error bound below the k-th, so every candidate that can reach the
// exact top-ke is among the kp), FP64 rescoring of the kp and the top-ke of
// those.  A query that fails the margin test makes the exact form return
// false after one synchronisation; the caller then reranks the batch in FP64.
static bool split_rerank(const Index& rq, const float* qu, uint64_t nq, uint32_t me, uint32_t ke, float inv_norm,
                         bool raw, Workspace& w, cudaStream_t st) {
  if (!rerank_tc_eligible(rq.dim, rq.bits)) return false;
  const uint32_t dim = rq.dim, bits = rq.bits, id_bits = bits_for(rq.n - 1);
  const uint8_t* codes = rq.codes.as<uint8_t>();
  const uint32_t* cand = w.sel_ids.as<uint32_t>();
  void* qs = w.q_split.ensure(nq * dim * 4);
  float* l1 = (float*)w.q_l1.ensure(nq * 4);
  launch_split_queries(qu, nq, dim, qs, l1, st);
  uint32_t* keys = (uint32_t*)w.keys2.ensure(nq * me * 4);
  launch_rerank_tc(codes, rq.n, dim, bits, qs, nq, cand, me, me, inv_norm, keys, w.tc_err_word(st), st);
  w.mark(st, 4);
  uint32_t* ok = w.out_keys.as<uint32_t>();
  uint32_t* oi = w.out_ids.as<uint32_t>();
  if (raw) {
    select_rows(w, keys, cand, nullptr, me, me, nq, ke, 32, id_bits, ok, oi, st);
    w.mark(st, 5);
    return true;
  }
  const uint32_t kp = std::min<uint32_t>(me, 2 * ke + 32);
  uint32_t* ck = (uint32_t*)w.rr_keys.ensure(nq * kp * 4);
  uint32_t* ci = (uint32_t*)w.rr_ids.ensure(nq * kp * 4);
  uint32_t* flag = (uint32_t*)w.rr_flag.ensure(4);
  uint32_t* flag_h = (uint32_t*)w.rr_flag_host.ensure(4);
  select_rows(w, keys, cand, nullptr, me, me, nq, kp, 32, id_bits, ck, ci, st);
  OVB_CUDA(cudaMemsetAsync(flag, 0, 4, st));
  launch_split_margin(ck, nq, kp, ke, l1, split_error_bound(dim, bits, inv_norm), flag, st);
  uint64_t* off = (uint64_t*)w.off.ensure((nq + 1) * 8);
  launch_uniform_offsets(off, nq, kp, st);
  uint32_t* k2 = (uint32_t*)w.rr_keys2.ensure(nq * kp * 4);
  launch_asym_subset(codes, dim, bits, qu, nq, off, ci, kp, inv_norm, k2, st);
  select_rows(w, k2, ci, nullptr, kp, kp, nq, ke, 32, id_bits, ok, oi, st);
  w.mark(st, 5);
  OVB_CUDA(cudaMemcpyAsync(flag_h, flag, 4, cudaMemcpyDeviceToHost, st));
  OVB_CUDA(cudaStreamSynchronize(st));
  return *flag_h == 0;
}

uint32_t engine_two_stage(const Index& rq, const Index& s1, const float* d_q, uint64_t nq,
                          uint64_t m, uint64_t k, Workspace& w, cudaStream_t st) {
  require_kind(rq, ORDVEC_INDEX_KIND_RANK_QUANT, "two-stage rerank");
  if (s1.dim != rq.dim) fail(ORDVEC_STATUS_DIM_MISMATCH, "stage-1 index dim must match RankQuant dim");
  if (s1.n != rq.n) fail(ORDVEC_STATUS_BAD_ARGUMENT, "stage-1 index len must match RankQuant len");
  const uint64_t m_req = m ? m : default_candidate_count(k, rq.n);
  w.mark(st, 0);
  if (!nq) return 0;
  const float* qu = normalised(w, d_q, nq, rq.dim, st);  // shared by both stages
  // the rerank reads the candidate set, not its order: stage 1 skips the sort
  struct Unordered {
    Workspace& w;
    explicit Unordered(Workspace& ws) : w(ws) { w.cand_unordered = true; }
    ~Unordered() { w.cand_unordered = false; }
  };
  uint32_t me;
  {
    Unordered guard(w);
    me = engine_candidates(s1, d_q, nq, m_req, nullptr, w, st, qu);
  }
  const uint32_t ke = (uint32_t)(k < me ? k : me);
  if (!ke) return ke;
  const float inv_norm = inv_rankquant_norm(rq.dim, rq.bits);
  uint32_t* ok = (uint32_t*)w.out_keys.ensure(nq * ke * 4);
  uint32_t* oi = (uint32_t*)w.out_ids.ensure(nq * ke * 4);
  const uint32_t id_bits = bits_for(rq.n - 1);
  const uint32_t* cand = w.sel_ids.as<uint32_t>();
  const uint32_t mode = rerank_mode(w, rq, nq, me, ke);
  if (mode != OVB_RERANK_FP64 && split_rerank(rq, qu, nq, me, ke, inv_norm, mode == OVB_RERANK_SPLIT_RAW, w, st))
    return ke;
  uint64_t* off = (uint64_t*)w.off.ensure((nq + 1) * 8);
  launch_uniform_offsets(off, nq, me, st);
  uint32_t* keys = (uint32_t*)w.keys2.ensure(nq * me * 4);
  launch_asym_subset(rq.codes.as<uint8_t>(), rq.dim, rq.bits, qu, nq, off, cand, me, inv_norm, keys, st);
  w.mark(st, 4);
  // rows are uniform (me candidates each): the strided form, not offsets
  select_rows(w, keys, cand, nullptr, me, me, nq, ke, 32, id_bits, ok, oi, st);
  w.mark(st, 5);
  return ke;
}

uint32_t engine_two_stage_ragged(const Index& rq, const Index& s1, const float* d_q, uint64_t nq,
                                 const uint64_t* m_of, uint64_t k, Workspace& w, cudaStream_t st) {
  require_kind(rq, ORDVEC_INDEX_KIND_RANK_QUANT, "two-stage rerank");
  if (s1.dim != rq.dim) fail(ORDVEC_STATUS_DIM_MISMATCH, "stage-1 index dim must match RankQuant dim");
  if (s1.n != rq.n) fail(ORDVEC_STATUS_BAD_ARGUMENT, "stage-1 index len must match RankQuant len");
  w.mark(st, 0);
  if (!nq || !k) return 0;
  uint64_t m_max = 0;
  for (uint64_t q = 0; q < nq; q++) m_max = std::max(m_max, m_of[q]);
  if (!m_max) return 0;
  const float* qu = normalised(w, d_q, nq, rq.dim, st);
  // ordered rows: each query's own top-m is the prefix of its top-m_max
  const uint32_t me = engine_candidates(s1, d_q, nq, m_max, nullptr, w, st, qu);
  const uint32_t ke = (uint32_t)(k < me ? k : me);
  if (!ke) return ke;
  uint64_t* h_off = (uint64_t*)w.off_host.ensure((nq + 1) * 8);
  OVB_CUDA(cudaStreamSynchronize(st));  // the pinned offsets may still feed an earlier copy
  h_off[0] = 0;
  for (uint64_t q = 0; q < nq; q++) h_off[q + 1] = h_off[q] + std::min<uint64_t>(m_of[q], me);
  uint64_t* off = (uint64_t*)w.off.ensure((nq + 1) * 8);
  OVB_CUDA(cudaMemcpyAsync(off, h_off, (nq + 1) * 8, cudaMemcpyHostToDevice, st));
  const uint64_t total = h_off[nq];
  uint32_t* cand = (uint32_t*)w.csr_ids.ensure(total * 4 + 4);
  launch_prefix_compact(w.sel_ids.as<uint32_t>(), me, off, nq, cand, st);
  uint32_t* keys = (uint32_t*)w.keys2.ensure(total * 4 + 4);
  launch_asym_subset(rq.codes.as<uint8_t>(), rq.dim, rq.bits, qu, nq, off, cand, me, inv_rankquant_norm(rq.dim, rq.bits),
                     keys, st);
  w.mark(st, 4);
  uint32_t* ok = (uint32_t*)w.out_keys.ensure(nq * ke * 4);
  uint32_t* oi = (uint32_t*)w.out_ids.ensure(nq * ke * 4);
  select_rows(w, keys, cand, off, 0, 0, nq, ke, 32, bits_for(rq.n - 1), ok, oi, st);
  w.mark(st, 5);
  return ke;
}

}  // namespace ovb
