// Shared pieces of the tensor-core scan kernels (scan_fastscan_tc.cu: one CTA
// per tile; scan_tc_pair.cu: persistent CTA pairs): the launch arguments, the
// FastScan score and bitmap keys of an integer accumulator, the accumulator
// thresholds of the filter epilogue, and the one-hot helpers of the builders.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ovb_common.cuh"

namespace ovb {
namespace tcs {

constexpr uint32_t kExactCompare = 0xFFFFFFFFu;  // amin: compare keys, not accumulators
constexpr uint32_t kNeverPasses = 0xFFFFFFFEu;   // amin past the tile's queries (acc < 2^23)

struct TcArgs {
  const uint8_t* blocks;  // FastScan device blocks, or bitmap rows (u64 words)
  uint64_t n;
  uint32_t pairs_pad;     // FastScan
  uint32_t qpv;           // bitmap: u64 words per row
  uint32_t n_top;         // bitmap: set bits per row (key = n_top - overlap)
  uint32_t key_kind;      // bitmap: 0 key = n_top - acc, 1 key = desc_key((float)acc), 2 Hamming
  const uint32_t* qpop;   // bitmap key_kind 2: popcount of each query's words
  uint32_t n_kb;          // 128-byte K-blocks
  uint32_t block_stride;
  const float* bias;
  const float* invq;
  float inv_norm;
  uint64_t nq;
  uint32_t nt;
  // dense output (keys != null)
  uint32_t* keys;
  uint64_t ld;
  // filter output
  const uint32_t* thr;
  const uint32_t* thr_pos;  // bitmap: sample position of the threshold (tie bound), or null
  uint32_t smp_stride;      // block stride of the sample the positions index
  uint64_t thr_stride;
  uint32_t* cnt;
  uint32_t cap;
  uint32_t* f_keys;
  uint32_t* f_ids;
  uint32_t* err;
  uint64_t expect_kept;  // filter: expected kept docs per query (0 = unknown)
};

// shl.b32 clamps shift amounts >= 32 to 32 (result 0); a "negative" amount
// wraps to a large unsigned one, so shl1(8 * nib - 32 * i) is the word i of the
// 16-byte one-hot row of nibble nib.
__device__ __forceinline__ uint32_t shl1(uint32_t amount) {
  uint32_t r;
  asm("shl.b32 %0, %1, %2;" : "=r"(r) : "r"(1u), "r"(amount));
  return r;
}

// Exact f32 value of an accumulator below 2^23 (acc <= 255 * pairs_pad): the
// integer is placed in the mantissa of 2^23 and 2^23 subtracted; no conversion
// instruction, same value as a round-to-nearest u32 -> f32 conversion.
__device__ __forceinline__ float acc_to_float(uint32_t acc) {
  return __fsub_rn(__uint_as_float(acc | 0x4B000000u), 8388608.0f);
}

// (bias + acc * inv_q) * inv_norm in f32, round-to-nearest at every step
// (src/fastscan.rs:306-307: raw = bias_sum + acc * inv_q, then * inv_norm), as
// the CUDA-core kernel computes it.
__device__ __forceinline__ float tc_score(uint32_t acc, float bias, float invq, float inv_norm) {
  return __fmul_rn(__fadd_rn(bias, __fmul_rn(acc_to_float(acc), invq)), inv_norm);
}

// Filter threshold on the accumulator.  With bias, inv_q, inv_norm finite,
// inv_q >= 0 and inv_norm > 0, every step of tc_score is monotone
// non-decreasing in acc (no NaN can arise), so desc_key(score) is non-increasing
// and {acc : key <= thr} = [amin, amax]; the binary search finds amin
// (amax + 1 when no accumulator passes).  Otherwise kExactCompare.
__device__ inline uint32_t filter_amin(float bias, float invq, float inv_norm, uint32_t thr, uint32_t amax) {
  if (!(isfinite(bias) && isfinite(invq) && isfinite(inv_norm) && invq >= 0.0f && inv_norm > 0.0f))
    return kExactCompare;
  uint32_t lo = 0, hi = amax + 1;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (desc_key(tc_score(mid, bias, invq, inv_norm)) <= thr)
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}


// Bitmap-mode key of an overlap accumulator (acc <= 64 * qpv < 2^24, so the
// f32 conversion is exact).
__device__ __forceinline__ uint32_t bm_key(const TcArgs& a, uint32_t acc) {
  return a.key_kind == 0 ? a.n_top - acc : desc_key(__uint2float_rn(acc));
}

// Smallest accumulator whose key is <= thr; both key kinds are strictly
// decreasing in acc, so key(acc) == thr exactly at acc == result when thr is
// the key of some row.
__device__ inline uint32_t bm_amin(const TcArgs& a, uint32_t thr) {
  if (a.key_kind == 0) return thr >= a.n_top ? 0u : a.n_top - thr;
  uint32_t lo = 0, hi = 64u * a.qpv + 1;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (bm_key(a, mid) <= thr)
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

// Sign bitmaps (key_kind 2): Hamming(q, d) = |q| + |d| - 2 |q AND d|.  The
// epilogue compares y = 2 acc + kHamBias - |d| (per doc row) against
// |q| + kHamBias - thr (per query), so the threshold test stays one compare
// per (doc, query) and key <= thr <=> y >= that bound.
constexpr uint32_t kHamBias = 1u << 20;

__device__ __forceinline__ uint32_t ham_y(uint32_t acc, uint32_t dpop) { return 2 * acc + kHamBias - dpop; }

// key of a (possibly transformed) accumulator for a query with popcount qpop
__device__ __forceinline__ uint32_t bm_key_q(const TcArgs& a, uint32_t qpop, uint32_t y) {
  return a.key_kind == 2 ? qpop + kHamBias - y : bm_key(a, y);
}

// smallest (transformed) accumulator whose key is <= thr
__device__ __forceinline__ uint32_t bm_amin_q(const TcArgs& a, uint32_t qpop, uint32_t thr) {
  return a.key_kind == 2 ? qpop + kHamBias - thr : bm_amin(a, thr);
}

// popcount of a bitmap row (qpv words), 0 for an invalid row
__device__ __forceinline__ uint32_t row_popcount(const TcArgs& a, uint64_t doc, bool valid) {
  uint32_t c = 0;
  if (valid) {
    const uint64_t* w = reinterpret_cast<const uint64_t*>(a.blocks) + doc * (uint64_t)a.qpv;
    for (uint32_t i = 0; i < a.qpv; i++) c += __popcll(__ldg(w + i));
  }
  return c;
}

__device__ __forceinline__ uint4 load_codes(const uint8_t* p) {
  uint4 v;
  asm volatile("ld.global.nc.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

// MODE 0: FastScan (A = one-hot of nibble codes, B = u8 LUTs, score by the
// FastScan formula).  MODE 1: bitmap AND-overlap (A = doc bits as 0/1 bytes,
// B = query bits as 0/1 bytes, acc = overlap, key = n_top - overlap).  MODE 2:
// the bitmap filter on FP4 tensor cores (A, B = bits as e2m1 nibbles of 1.0 /
// 0, f32 acc = overlap), CTA pairs only.
}  // namespace tcs

// Forms of the tensor-core scans: one CTA per 256-doc tile (scan_fastscan_tc.cu),
// and the persistent forms of scan_tc_pair.cu: one CTA per SM, or CTA pairs.
enum class TcForm { kTile, kPersist, kPair };
TcForm tc_form(int mode);  // MODE 0 FastScan, 1 bitmap
uint32_t tc_persist_seg_cap();
uint32_t tc_fp4_max_words();  // longest bitmap row (u64 words) of the FP4 form
// b_rows = the query operand; pair: CTA pairs, else one CTA per SM
template <int MODE>
void launch_tc_pair(tcs::TcArgs a, const uint8_t* b_rows, cudaStream_t stream, bool pair);

}  // namespace ovb
