// K4 / K5: asymmetric RankQuant scoring against the float query.
//
// score(q, d) = sum_j q_unit[j] * bucket_centre(code_j) * inv_norm
// (src/quant.rs:697-847, src/quant_kernels.rs:23-581; subset rerank
// src/quant.rs:1126-1281).  The reference's float scores are not bit-stable
// across its own SIMD tiers (docs/determinism.md), so this path is checked
// against an FP64 oracle within 1e-5 relative; ids break ties by global row id.
//
// Decoding: a document row is `bpv` bytes, MSB-first codes (src/rank.rs:128).
// A group of G lanes (16 or 32) reads one row as u32 words (lane g takes words
// g, g+G, ...), so a warp instruction reads 32/G consecutive rows; the query
// coordinates of a lane's words never change across rows and live in
// registers.  Each code becomes its exact centred value without an int->float
// conversion: f = as_float(0x3F800000 | code << (23-B)) = 1 + code/2^B, then
// f * 2^B - (2^B + (2^B-1)/2) = code - (2^B-1)/2, then one FMA with q.
#include "ovb_common.cuh"
#include "ovb_kernels.h"

namespace ovb {

namespace {

constexpr int kThreads = 256;

// Dot product of one u32 word of codes with its query slice.  Each of the CPB
// code positions of a byte keeps its own FP32 chain of 4 products (short
// chains keep the rounding error per chain tiny); the chains are combined in
// FP64 so the cross-word sum meets the 1e-5-relative-of-FP64 contract even for
// scores near zero, where FP32 cancellation would not.
template <int BITS>
__device__ __forceinline__ double word_dot(uint32_t x, const float* q) {
  constexpr int CPB = 8 / BITS;
  constexpr uint32_t MASK = (1u << BITS) - 1;
  constexpr float SCALE = (float)(1u << BITS);
  constexpr float OFF = -((float)(1u << BITS) + ((float)(1u << BITS) - 1.0f) * 0.5f);
  float a[CPB];
#pragma unroll
  for (int i = 0; i < CPB; i++) a[i] = 0.0f;
#pragma unroll
  for (int b = 0; b < 4; b++) {
#pragma unroll
    for (int i = 0; i < CPB; i++) {
      const int s = 8 * b + 8 - BITS * (i + 1);
      const uint32_t code = (x >> s) & MASK;
      const float f = __uint_as_float(0x3F800000u | (code << (23 - BITS)));
      const float c = fmaf(f, SCALE, OFF);
      a[i] = fmaf(q[b * CPB + i], c, a[i]);
    }
  }
  double t = 0.0;
#pragma unroll
  for (int i = 0; i < CPB; i++) t += (double)a[i];
  return t;
}

__device__ __forceinline__ uint32_t score_key(double dot, float inv_norm) {
  return desc_key((float)(dot * (double)inv_norm));
}

// G lanes per row, W words per lane (compile time), q in registers.
template <int BITS, int G, int W>
__device__ __forceinline__ void load_q(const float* qu, uint32_t words, int g, float (&qr)[W][32 / BITS]) {
  constexpr int CPW = 32 / BITS;
#pragma unroll
  for (int i = 0; i < W; i++) {
    const uint32_t w = g + i * G;
#pragma unroll
    for (int c = 0; c < CPW; c++) qr[i][c] = w < words ? qu[w * CPW + c] : 0.0f;
  }
}

template <int BITS, int G, int W>
__device__ __forceinline__ double row_dot(const uint32_t* row, uint32_t words, int g,
                                          const float (&qr)[W][32 / BITS]) {
  double acc = 0.0;
#pragma unroll
  for (int i = 0; i < W; i++) {
    const uint32_t w = g + i * G;
    if (w < words) acc += word_dot<BITS>(__ldcs(row + w), qr[i]);
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
  return acc;
}

template <int BITS, int G, int W>
__global__ void __launch_bounds__(kThreads)
    asym_scan_kernel(const uint8_t* __restrict__ codes, uint64_t n, uint32_t dim,
                     const float* __restrict__ q_unit, float inv_norm,
                     uint32_t* __restrict__ keys, uint64_t ld) {
  constexpr int RPW = 32 / G;  // rows per warp instruction
  const uint64_t qi = blockIdx.y;
  const uint32_t words = dim * BITS / 32;
  const int lane = threadIdx.x & 31, g = lane % G;
  float qr[W][32 / BITS];
  load_q<BITS, G, W>(q_unit + qi * dim, words, g, qr);
  const uint64_t gw = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kThreads / 32;
  uint32_t* out = keys + qi * ld;
  for (uint64_t base = gw * RPW; base < n; base += nw * RPW) {
    const uint64_t doc = base + lane / G;
    const uint64_t rd = doc < n ? doc : n - 1;
    const double dot = row_dot<BITS, G, W>((const uint32_t*)codes + rd * words, words, g, qr);
    if (g == 0 && doc < n) out[doc] = score_key(dot, inv_norm);
  }
}

template <int BITS, int G, int W>
__global__ void __launch_bounds__(kThreads)
    asym_subset_kernel(const uint8_t* __restrict__ codes, uint32_t dim,
                       const float* __restrict__ q_unit, const uint64_t* __restrict__ off,
                       const uint32_t* __restrict__ cands, float inv_norm,
                       uint32_t* __restrict__ keys) {
  constexpr int RPW = 32 / G;
  const uint64_t qi = blockIdx.y;
  const uint64_t s = off[qi], e = off[qi + 1];
  const uint32_t words = dim * BITS / 32;
  const int lane = threadIdx.x & 31, g = lane % G;
  float qr[W][32 / BITS];
  load_q<BITS, G, W>(q_unit + qi * dim, words, g, qr);
  const uint64_t gw = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kThreads / 32;
  for (uint64_t base = s + gw * RPW; base < e; base += nw * RPW) {
    const uint64_t i = base + lane / G;
    const uint64_t ri = i < e ? i : e - 1;
    const double dot = row_dot<BITS, G, W>((const uint32_t*)codes + (uint64_t)cands[ri] * words, words, g, qr);
    if (g == 0 && i < e) keys[i] = score_key(dot, inv_norm);
  }
}

// Generic byte-wise path for rows that are not a whole number of u32 words or
// too wide for the register path: one warp per row, q read from global.
__device__ __forceinline__ double generic_row_dot(const uint8_t* row, uint32_t dim, uint32_t bits,
                                                  const float* qu) {
  const int lane = threadIdx.x & 31;
  const uint32_t cpb = 8 / bits, mask = (1u << bits) - 1;
  const double centre = ((double)(1u << bits) - 1.0) * 0.5;
  double acc = 0.0;
  for (uint32_t j = lane; j < dim; j += 32) {
    const uint32_t code = (row[j / cpb] >> ((cpb - 1 - j % cpb) * bits)) & mask;
    acc = fma((double)qu[j], (double)code - centre, acc);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
  return acc;
}

__global__ void __launch_bounds__(kThreads)
    asym_scan_generic(const uint8_t* __restrict__ codes, uint64_t n, uint32_t dim, uint32_t bits,
                      const float* __restrict__ q_unit, float inv_norm,
                      uint32_t* __restrict__ keys, uint64_t ld) {
  const uint64_t qi = blockIdx.y;
  const uint32_t bpv = dim * bits / 8;
  const uint64_t gw = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kThreads / 32;
  for (uint64_t doc = gw; doc < n; doc += nw) {
    const double dot = generic_row_dot(codes + doc * bpv, dim, bits, q_unit + qi * dim);
    if ((threadIdx.x & 31) == 0) keys[qi * ld + doc] = score_key(dot, inv_norm);
  }
}

__global__ void __launch_bounds__(kThreads)
    asym_subset_generic(const uint8_t* __restrict__ codes, uint32_t dim, uint32_t bits,
                        const float* __restrict__ q_unit, const uint64_t* __restrict__ off,
                        const uint32_t* __restrict__ cands, float inv_norm,
                        uint32_t* __restrict__ keys) {
  const uint64_t qi = blockIdx.y;
  const uint32_t bpv = dim * bits / 8;
  const uint64_t gw = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kThreads / 32;
  for (uint64_t i = off[qi] + gw; i < off[qi + 1]; i += nw) {
    const double dot = generic_row_dot(codes + (uint64_t)cands[i] * bpv, dim, bits, q_unit + qi * dim);
    if ((threadIdx.x & 31) == 0) keys[i] = score_key(dot, inv_norm);
  }
}

unsigned grid_x(uint64_t rows_per_cta, uint64_t n) {
  uint64_t g = (n + rows_per_cta - 1) / rows_per_cta;
  if (g < 1) g = 1;
  if (g > 148 * 8) g = 148 * 8;
  return (unsigned)g;
}

// Register path is used when rows are whole u32 words and a lane holds at
// most 8 words (<= 128 query floats in registers).
struct Plan {
  bool fast;
  int G, W;
};
Plan plan_for(uint32_t dim, uint32_t bits) {
  if ((dim * bits) % 32 != 0) return {false, 0, 0};
  uint32_t words = dim * bits / 32;
  int G = words <= 128 ? 16 : 32;
  uint32_t W = (words + G - 1) / G;
  if (W > 8 || W * (32 / bits) > 128) return {false, 0, 0};
  int Wp = W <= 1 ? 1 : W <= 2 ? 2 : W <= 4 ? 4 : 8;
  return {true, G, Wp};
}

template <int BITS, int G>
void dispatch_w(int W, bool subset, dim3 grid, cudaStream_t st, const uint8_t* codes, uint64_t n,
                uint32_t dim, const float* qu, float inv_norm, uint32_t* keys, uint64_t ld,
                const uint64_t* off, const uint32_t* cands) {
#define OVB_ASYM_CASE(WV)                                                                        \
  if (W == WV) {                                                                                 \
    if (subset)                                                                                  \
      asym_subset_kernel<BITS, G, WV><<<grid, kThreads, 0, st>>>(codes, dim, qu, off, cands, inv_norm, keys); \
    else                                                                                         \
      asym_scan_kernel<BITS, G, WV><<<grid, kThreads, 0, st>>>(codes, n, dim, qu, inv_norm, keys, ld); \
    return;                                                                                      \
  }
  OVB_ASYM_CASE(1)
  OVB_ASYM_CASE(2)
  OVB_ASYM_CASE(4)
  if constexpr (BITS != 1) {
    OVB_ASYM_CASE(8)
  }
#undef OVB_ASYM_CASE
}

template <int BITS>
void dispatch_g(const Plan& p, bool subset, dim3 grid, cudaStream_t st, const uint8_t* codes,
                uint64_t n, uint32_t dim, const float* qu, float inv_norm, uint32_t* keys,
                uint64_t ld, const uint64_t* off, const uint32_t* cands) {
  if (p.G == 16)
    dispatch_w<BITS, 16>(p.W, subset, grid, st, codes, n, dim, qu, inv_norm, keys, ld, off, cands);
  else
    dispatch_w<BITS, 32>(p.W, subset, grid, st, codes, n, dim, qu, inv_norm, keys, ld, off, cands);
}

void dispatch(uint32_t bits, const Plan& p, bool subset, dim3 grid, cudaStream_t st,
              const uint8_t* codes, uint64_t n, uint32_t dim, const float* qu, float inv_norm,
              uint32_t* keys, uint64_t ld, const uint64_t* off, const uint32_t* cands) {
  if (bits == 1)
    dispatch_g<1>(p, subset, grid, st, codes, n, dim, qu, inv_norm, keys, ld, off, cands);
  else if (bits == 2)
    dispatch_g<2>(p, subset, grid, st, codes, n, dim, qu, inv_norm, keys, ld, off, cands);
  else
    dispatch_g<4>(p, subset, grid, st, codes, n, dim, qu, inv_norm, keys, ld, off, cands);
}

}  // namespace

void launch_asym_scan(const uint8_t* codes, uint64_t n, uint32_t dim, uint32_t bits,
                      const float* q_unit, uint64_t nq, float inv_norm, uint32_t* keys,
                      uint64_t ld, cudaStream_t stream) {
  if (!n || !nq) return;
  const Plan p = plan_for(dim, bits);
  for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
    unsigned gy = (unsigned)((nq - q0) < 65535 ? (nq - q0) : 65535);
    if (p.fast) {
      dim3 grid(grid_x((kThreads / 32) * (32 / p.G), n), gy);
      dispatch(bits, p, false, grid, stream, codes, n, dim, q_unit + q0 * dim, inv_norm, keys + q0 * ld, ld,
               nullptr, nullptr);
    } else {
      dim3 grid(grid_x(kThreads / 32, n), gy);
      asym_scan_generic<<<grid, kThreads, 0, stream>>>(codes, n, dim, bits, q_unit + q0 * dim, inv_norm,
                                                       keys + q0 * ld, ld);
    }
    launched();
  }
}

void launch_asym_subset(const uint8_t* codes, uint32_t dim, uint32_t bits, const float* q_unit,
                        uint64_t nq, const uint64_t* offsets, const uint32_t* cands,
                        uint64_t max_row, float inv_norm, uint32_t* keys, cudaStream_t stream) {
  if (!nq || !max_row) return;
  const Plan p = plan_for(dim, bits);
  for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
    unsigned gy = (unsigned)((nq - q0) < 65535 ? (nq - q0) : 65535);
    if (p.fast) {
      dim3 grid(grid_x((kThreads / 32) * (32 / p.G), max_row), gy);
      dispatch(bits, p, true, grid, stream, codes, 0, dim, q_unit + q0 * dim, inv_norm, keys, 0,
               offsets + q0, cands);
    } else {
      dim3 grid(grid_x(kThreads / 32, max_row), gy);
      asym_subset_generic<<<grid, kThreads, 0, stream>>>(codes, dim, bits, q_unit + q0 * dim, offsets + q0,
                                                         cands, inv_norm, keys);
    }
    launched();
  }
}

}  // namespace ovb
