// Host-side launch interface of the sm_100a kernels.  All pointers are
// device pointers; every launch is asynchronous on `stream`.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstddef>

namespace ovb {

// ---- K7 select (select.cu) ---------------------------------------------------
constexpr uint32_t kSelectSmemCap = 4096;  // k up to this sorts in shared memory

struct SelectArgs {
  const uint32_t* keys;     // row r at keys + r*ld (or + row_off[r])
  const uint32_t* ids;      // explicit global ids (same layout) or null = position
  const uint64_t* row_off;  // ragged rows (rows+1 offsets) or null = uniform n
  uint64_t ld;
  uint64_t n;
  uint32_t k;         // output stride; each row keeps min(k, n_row), rest sentinel
  uint32_t key_bits;  // significant bits of key32
  uint32_t id_bits;   // significant bits of id32
  uint32_t* out_keys;
  uint32_t* out_ids;
  const uint32_t* row_len;  // optional: row r holds min(row_len[r], n) entries at r*ld
  uint32_t unordered;       // 1: a row's k_eff winners in any order (the set only; per-row and cluster forms)
};
// u64 scratch elements launch_select_rows may use for `rows` rows of length n
// (0 for ragged rows): global sort buffers for k > kSelectSmemCap, and the
// whole-GPU form's histograms and winners for a few rows of >= 2^20 keys.
size_t select_rows_scratch_elems(uint64_t rows, uint32_t k, uint64_t n);
void launch_select_rows(const SelectArgs& a, uint64_t rows, uint64_t* scratch,
                        cudaStream_t stream);

// ---- K8 query preparation (prep.cu) ------------------------------------------
void launch_l2_normalise(const float* q, uint64_t nq, uint32_t dim, float* out,
                         cudaStream_t stream);
void launch_sign_query(const float* q, uint64_t nq, uint32_t dim, uint64_t* out,
                       cudaStream_t stream);
void launch_bitmap_query(const float* q, uint64_t nq, uint32_t dim, uint32_t n_top,
                         uint64_t* out, cudaStream_t stream);
void launch_fastscan_lut(const float* q_unit, uint64_t nq, uint32_t dim, uint32_t pairs_pad,
                         uint8_t* lut, float* bias_sum, float* inv_q, cudaStream_t stream);

// ---- K1/K2/K6 popcount scans (scan_popc.cu) -> key32 [nq][ld] ------------------
// mode 0: sign Hamming (key = hamming); mode 1: bitmap AND overlap
// (key = n_top - overlap).
void launch_popc_scan(int mode, const uint64_t* words, uint64_t n, uint32_t qpv,
                      const uint64_t* qbits, uint64_t nq, uint32_t n_top, uint32_t* keys,
                      uint64_t ld, cudaStream_t stream);
// Subset form: key32 for CSR candidate entries (keys share the CSR layout).
void launch_popc_subset(int mode, const uint64_t* words, uint32_t qpv, const uint64_t* qbits,
                        uint64_t nq, const uint64_t* offsets, const uint32_t* cands,
                        uint64_t max_row, uint32_t n_top, uint32_t* keys, cudaStream_t stream);
// Multi-bucket bilinear score (desc float key).
void launch_multibucket_scan(const uint64_t* words, uint64_t n, uint32_t qpb, uint32_t nb,
                             const uint64_t* qbits, const float* w, uint64_t nq,
                             uint32_t* keys, uint64_t ld, cudaStream_t stream);
void launch_multibucket_query(const float* q, uint64_t nq, uint32_t dim, uint32_t bits,
                              uint64_t* out, cudaStream_t stream);

// ---- K3 FastScan (scan_fastscan.cu) --------------------------------------------
void launch_fastscan_scan(const uint8_t* blocks, uint64_t n, uint32_t pairs_pad,
                          const uint8_t* lut, const float* bias_sum, const float* inv_q,
                          float inv_norm, uint64_t nq, uint32_t* keys, uint64_t ld,
                          cudaStream_t stream);
// Tensor-core form (scan_fastscan_tc.cu): same keys, bit for bit; *err (device
// u32) gets bit 0 set if a bounded wait timed out.  block_stride > 1 scores
// only every block_stride-th 32-doc block; keys[q][u] then holds the u-th
// sampled doc (fastscan_tc_sample_docs columns).
void launch_fastscan_scan_tc(const uint8_t* blocks, uint64_t n, uint32_t pairs_pad, const uint8_t* lut,
                             const float* bias_sum, const float* inv_q, float inv_norm, uint64_t nq,
                             uint32_t block_stride, uint32_t* keys, uint64_t ld, uint32_t* err,
                             cudaStream_t stream);
uint64_t fastscan_tc_sample_docs(uint64_t n, uint32_t block_stride);
// Threshold filter: appends (key32, doc) with key32 <= thr[q * thr_stride] to
// row q of f_keys / f_ids (capacity cap); cnt[q] (zeroed by the caller) counts
// every qualifying doc.  expect_kept: the expected count per query (picks the
// kernel form whose kept-entry lists fit it; 0 = unknown).
void launch_fastscan_filter_tc(const uint8_t* blocks, uint64_t n, uint32_t pairs_pad, const uint8_t* lut,
                               const float* bias_sum, const float* inv_q, float inv_norm, uint64_t nq,
                               const uint32_t* thr, uint64_t thr_stride, uint32_t* cnt, uint32_t cap,
                               uint32_t* f_keys, uint32_t* f_ids, uint64_t expect_kept, uint32_t* err,
                               cudaStream_t stream);
// Tensor-core bitmap overlap scan (same file, u8 x u8 -> s32 on 0/1 bytes).
// Rows of qpv u64 words; key_kind 0: key32 = n_top - popcount(q AND d)
// (constant-weight bitmap), 1: key32 = desc_key((float)popcount) (multi-bucket
// with identity weights), 2: key32 = popcount(q XOR d) = |q| + |d| - 2 |q AND d|
// (sign bitmap; qpop = |q| per query).  The query operand is the query bits
// expanded to 0/1 bytes (launch_bitmap_tc_query, which also writes qpop when
// given), bitmap_tc_kblocks(qpv) * 128 per query.
uint32_t bitmap_tc_kblocks(uint32_t qpv);
void launch_bitmap_tc_query(const uint64_t* qbits, uint64_t nq, uint32_t qpv, uint8_t* out, uint32_t* qpop,
                            cudaStream_t stream);
void launch_bitmap_scan_tc(const uint64_t* words, uint64_t n, uint32_t qpv, uint32_t key_kind, uint32_t n_top,
                           const uint32_t* qpop, const uint8_t* q_bytes, uint64_t nq, uint32_t block_stride,
                           uint32_t* keys, uint64_t ld, uint32_t* err, cudaStream_t stream);
// The same scan on FP4 tensor cores (kind::mxf4): the query operand is the
// query bits as packed e2m1 nibbles (launch_bitmap_fp4_query),
// bitmap_fp4_kblocks(qpv) * 128 bytes per query; bitmap_fp4_usable(qpv) says
// whether the filter below may take it (OVB_BITMAP_FP4=0 says no).
uint32_t bitmap_fp4_kblocks(uint32_t qpv);
bool bitmap_fp4_usable(uint32_t qpv);
void launch_bitmap_fp4_query(const uint64_t* qbits, uint64_t nq, uint32_t qpv, uint8_t* out, cudaStream_t stream);
// Filter with a tie bound: keeps (key32, doc) <= (thr, tdoc) in (key, doc)
// order, tdoc = the doc of sample position thr_pos[q * thr_stride] of a sample
// taken with block stride smp_stride (every doc at key < thr when thr_pos is null).
// With q_nib (the FP4 query operand) it runs on the FP4 tensor cores, else on
// int8 ones with q_bytes; same results.
void launch_bitmap_filter_tc(const uint64_t* words, uint64_t n, uint32_t qpv, uint32_t key_kind, uint32_t n_top,
                             const uint32_t* qpop, const uint8_t* q_bytes, const uint8_t* q_nib, uint64_t nq,
                             const uint32_t* thr, const uint32_t* thr_pos, uint32_t smp_stride, uint64_t thr_stride,
                             uint32_t* cnt, uint32_t cap, uint32_t* f_keys, uint32_t* f_ids, uint32_t* err,
                             cudaStream_t stream);
// *flag |= 1 when some cnt[q] < need or > cap.
void launch_filter_check(const uint32_t* cnt, uint64_t nq, uint32_t need, uint32_t cap, uint32_t* flag,
                         cudaStream_t stream);
void launch_fastscan_relayout(const uint8_t* ref_blocks, uint64_t n, uint32_t pairs,
                              uint32_t pairs_pad, uint8_t* dev_blocks, cudaStream_t stream);

// ---- K4-TC split-BF16 asymmetric scan on tcgen05 (scan_rank_tc.cu) -------------
bool rank_tc_eligible(uint32_t dim, uint32_t bits);
// |split score - exact score| <= split_error_bound(...) * |q_unit|_1
float split_error_bound(uint32_t dim, uint32_t bits, float inv_norm);
// q_unit rows -> [2 nq x dim] bf16 (row 2i = hi, 2i+1 = lo) and |q|_1 per row
void launch_split_queries(const float* q_unit, uint64_t nq, uint32_t dim, void* out_bf16, float* l1,
                          cudaStream_t stream);
// keys[q][u] (ld) = desc key of the split-BF16 score of logical doc u; with
// block_stride > 1 only every block_stride-th 32-doc block is scored (u = the
// sampled doc's position, fastscan_tc_sample_docs columns); q_per_tile 0 = default
void launch_rank_scan_tc(const uint8_t* codes, uint64_t n, uint32_t dim, uint32_t bits, const void* q_split,
                         uint64_t nq, float inv_norm, uint32_t block_stride, uint32_t* keys, uint64_t ld,
                         uint32_t q_per_tile, uint32_t* err, cudaStream_t stream);
// Threshold filter: appends (key32, doc) with key32 <= thr[q * thr_stride] to
// row q of f_keys / f_ids (capacity cap); cnt[q] (zeroed by the caller) counts
// every qualifying doc (bit 31 set when a tile's list overflowed).
void launch_rank_filter_tc(const uint8_t* codes, uint64_t n, uint32_t dim, uint32_t bits, const void* q_split,
                           uint64_t nq, float inv_norm, const uint32_t* thr, uint64_t thr_stride, uint32_t* cnt,
                           uint32_t cap, uint32_t* f_keys, uint32_t* f_ids, uint32_t q_per_tile, uint32_t* err,
                           cudaStream_t stream);
// flag |= 1 if some row's kp-th key is not below its k-th minus twice the bound
void launch_split_margin(const uint32_t* sel_keys, uint64_t nq, uint32_t kp, uint32_t k, const float* l1,
                         float bound_per_l1, uint32_t* flag, cudaStream_t stream);

// ---- K5-TC split-BF16 candidate rerank on tcgen05 (rerank_tc.cu) ---------------
// dim % 64 == 0 and 16 <= dim * bits / 8 <= 256, a multiple of 16
bool rerank_tc_eligible(uint32_t dim, uint32_t bits);
// keys[q * ld + j] = desc key of the split-BF16 score of candidate cands[q * ld + j], j < m
void launch_rerank_tc(const uint8_t* codes, uint64_t n, uint32_t dim, uint32_t bits, const void* q_split,
                      uint64_t nq, const uint32_t* cands, uint64_t ld, uint32_t m, float inv_norm, uint32_t* keys,
                      uint32_t* err, cudaStream_t stream);

// ---- self-test (selftest.cu): out[0] = 1 when a bounded mbarrier wait on a
// barrier nothing arrives at gave up, out[1..2] = the nanoseconds it waited
void launch_wait_probe(uint32_t* d_out, cudaStream_t stream);

// ---- K9 Rank (u16) index scans (scan_rank_full.cu) -> key32 [nq][ld] ------------
float rank_norm_f32(uint32_t dim);
// Rank::search: q_ranks = the queries' u16 ranks (nq x dim)
void launch_rank_sym_scan(const uint16_t* ranks, uint64_t n, uint32_t dim, const uint16_t* q_ranks, uint64_t nq,
                          uint32_t* keys, uint64_t ld, cudaStream_t stream);
// Rank::search_asymmetric: q_unit rows; q_sum (nq floats) is scratch the launch fills
void launch_rank_asym_scan(const uint16_t* ranks, uint64_t n, uint32_t dim, const float* q_unit, float* q_sum,
                           uint64_t nq, uint32_t* keys, uint64_t ld, cudaStream_t stream);

// ---- K4/K5 asymmetric RankQuant scoring (scan_asym.cu) ---------------------------
void launch_asym_scan(const uint8_t* codes, uint64_t n, uint32_t dim, uint32_t bits,
                      const float* q_unit, uint64_t nq, float inv_norm, uint32_t* keys,
                      uint64_t ld, cudaStream_t stream);
void launch_asym_subset(const uint8_t* codes, uint32_t dim, uint32_t bits, const float* q_unit,
                        uint64_t nq, const uint64_t* offsets, const uint32_t* cands,
                        uint64_t max_row, float inv_norm, uint32_t* keys, cudaStream_t stream);

// ---- encoders (encode.cu) ----------------------------------------------------------
// kind: 0 RankQuant packed codes, 1 sign bitmap, 2 const-weight bitmap, 3 FastScan
// (device layout), 4 multi-bucket bitmaps.
void launch_encode(int kind, const float* vecs, uint64_t n, uint32_t dim, uint32_t bits,
                   uint32_t n_top, uint32_t pairs_pad, void* out, uint64_t first_doc,
                   cudaStream_t stream);
uint32_t fastscan_pairs_pad(uint32_t dim);
uint64_t fastscan_block_bytes(uint32_t pairs_pad);

// sets *flag (device u32, caller-zeroed) if any value is non-finite
void launch_finite_flag(const float* x, uint64_t count, uint32_t* flag, cudaStream_t stream);

// helper: key32 -> float score / sentinel mapping and uniform offsets
void launch_uniform_offsets(uint64_t* off, uint64_t nq, uint64_t m, cudaStream_t stream);
// CSR rows from prefixes: row q of dst (at off[q]) = the first off[q+1] - off[q]
// entries of row q of src (row stride ld)
void launch_prefix_compact(const uint32_t* src, uint64_t ld, const uint64_t* off, uint64_t nq, uint32_t* dst,
                           cudaStream_t stream);
// ids[i] >= n (sentinels of underfull select rows) -> 0, so a gather stays in bounds
void launch_clamp_ids(uint32_t* ids, uint64_t count, uint32_t n, cudaStream_t stream);
void launch_keys_to_results(const uint32_t* keys, const uint32_t* ids, uint64_t count,
                            int mode, uint32_t n_top, float* scores, int64_t* out_ids,
                            cudaStream_t stream);

}  // namespace ovb
