// K4 / K5: asymmetric RankQuant scoring against the float query.
//
// score(q, d) = sum_j q_unit[j] * bucket_centre(code_j) * inv_norm
// (src/quant.rs:697-847, src/quant_kernels.rs:23-581; subset rerank
// src/quant.rs:1126-1281).  The reference's float scores are not bit-stable
// across its own SIMD tiers (docs/determinism.md), so this path is checked
// against an FP64 oracle within 1e-5 relative (floor 1e-3); ids break ties by
// global row id.
//
// Arithmetic (exact to ~1e-14): with f_j = 1 + code_j / 2^B,
//   sum_j q_j (code_j - c) = sum_j (q_j 2^B) f_j - (2^B + c) sum_j q_j,  c = (2^B-1)/2.
// f_j is built directly as a double from the code bits (high word
// 0x3FF00000 | code << (20-B)), q_j 2^B is held as a double in registers, and
// each code costs one DFMA whose product is exact (24 + 5 significant bits), so
// the only rounding is the FP64 accumulation.
//
// Decoding: a row is `bpv` bytes, MSB-first codes (src/rank.rs:128), read as
// u32 words by a full warp (lane l takes words l, l+32, ...): every warp load
// is 128 contiguous bytes and each lane's query coordinates never change
// across rows.
#include <cstdlib>

#include "ovb_common.cuh"
#include "ovb_kernels.h"

namespace ovb {

namespace {

constexpr int kThreads = 256;

// Four independent DFMA chains per lane (code c of a word goes to chain c % 4)
// so consecutive DFMAs do not wait on each other.
template <int BITS>
__device__ __forceinline__ void word_dot(uint32_t x, const double* qs, double (&acc)[4]) {
  constexpr int CPB = 8 / BITS;
  constexpr uint32_t MASK = (1u << BITS) - 1;
#pragma unroll
  for (int b = 0; b < 4; b++) {
#pragma unroll
    for (int i = 0; i < CPB; i++) {
      const int s = 8 * b + 8 - BITS * (i + 1);
      const uint32_t code = (x >> s) & MASK;
      const double f = __hiloint2double((int)(0x3FF00000u | (code << (20 - BITS))), 0);
      acc[(b * CPB + i) & 3] = fma(qs[b * CPB + i], f, acc[(b * CPB + i) & 3]);
    }
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}

// q slice of this lane as q * 2^B (doubles) and the warp-wide sum of q.
template <int BITS, int W>
__device__ __forceinline__ double load_q(const float* qu, uint32_t words, int lane,
                                         double (&qs)[W][32 / BITS]) {
  constexpr int CPW = 32 / BITS;
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < W; i++) {
    const uint32_t w = lane + i * 32;
#pragma unroll
    for (int c = 0; c < CPW; c++) {
      const double v = w < words ? (double)qu[w * CPW + c] : 0.0;
      s += v;
      qs[i][c] = v * (double)(1u << BITS);
    }
  }
  return warp_sum(s);
}

// This lane's words of a row (lane + 32 i); zero past the row.
template <int W>
__device__ __forceinline__ void load_row(const uint32_t* row, uint32_t words, int lane, uint32_t (&x)[W]) {
#pragma unroll
  for (int i = 0; i < W; i++) {
    const uint32_t w = lane + i * 32;
    x[i] = w < words ? __ldg(row + w) : 0u;
  }
}

// Zero words (and the zero query coordinates past the row) add exact zeros.
template <int BITS, int W>
__device__ __forceinline__ double words_dot(const uint32_t (&x)[W], const double (&qs)[W][32 / BITS]) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < W; i++) word_dot<BITS>(x[i], qs[i], acc);
  return warp_sum((acc[0] + acc[1]) + (acc[2] + acc[3]));
}

template <int BITS, int W>
__device__ __forceinline__ double row_dot(const uint32_t* row, uint32_t words, int lane,
                                          const double (&qs)[W][32 / BITS]) {
  uint32_t x[W];
  load_row<W>(row, words, lane, x);
  return words_dot<BITS, W>(x, qs);
}

template <int BITS>
__device__ __forceinline__ uint32_t finish(double dot, double qsum, float inv_norm) {
  constexpr double OFF = (double)(1u << BITS) + ((double)(1u << BITS) - 1.0) * 0.5;
  return desc_key((float)((dot - OFF * qsum) * (double)inv_norm));
}

template <int BITS, int W>
__global__ void __launch_bounds__(kThreads)
    asym_scan_kernel(const uint8_t* __restrict__ codes, uint64_t n, uint32_t dim,
                     const float* __restrict__ q_unit, float inv_norm,
                     uint32_t* __restrict__ keys, uint64_t ld) {
  const uint64_t qi = blockIdx.y;
  const uint32_t words = dim * BITS / 32;
  const int lane = threadIdx.x & 31;
  double qs[W][32 / BITS];
  const double qsum = load_q<BITS, W>(q_unit + qi * dim, words, lane, qs);
  const uint64_t gw = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kThreads / 32;
  uint32_t* out = keys + qi * ld;
  for (uint64_t doc = gw; doc < n; doc += nw) {
    const double dot = row_dot<BITS, W>((const uint32_t*)codes + doc * words, words, lane, qs);
    if (lane == 0) out[doc] = finish<BITS>(dot, qsum, inv_norm);
  }
}

template <int BITS, int W>
__global__ void __launch_bounds__(kThreads)
    asym_subset_kernel(const uint8_t* __restrict__ codes, uint32_t dim,
                       const float* __restrict__ q_unit, const uint64_t* __restrict__ off,
                       const uint32_t* __restrict__ cands, float inv_norm,
                       uint32_t* __restrict__ keys) {
  const uint64_t qi = blockIdx.y;
  const uint64_t s = off[qi], e = off[qi + 1];
  const uint32_t words = dim * BITS / 32;
  const int lane = threadIdx.x & 31;
  double qs[W][32 / BITS];
  const double qsum = load_q<BITS, W>(q_unit + qi * dim, words, lane, qs);
  const uint64_t gw = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kThreads / 32;
  // software pipeline: the next row's candidate id and words are in flight
  // while this row is scored
  const uint32_t* rows = (const uint32_t*)codes;
  uint64_t i = s + gw;
  if (i >= e) return;
  uint32_t x[W];
  load_row<W>(rows + (uint64_t)cands[i] * words, words, lane, x);
  uint32_t next_id = i + nw < e ? cands[i + nw] : 0u;
  for (; i < e; i += nw) {
    uint32_t y[W];
    const bool more = i + nw < e;
    if (more) load_row<W>(rows + (uint64_t)next_id * words, words, lane, y);
    if (i + 2 * nw < e) next_id = cands[i + 2 * nw];
    const double dot = words_dot<BITS, W>(x, qs);
    if (lane == 0) keys[i] = finish<BITS>(dot, qsum, inv_norm);
    if (more) {
#pragma unroll
      for (int k = 0; k < W; k++) x[k] = y[k];
    }
  }
}

// Generic path for rows that are not whole u32 words or wider than the
// register path: one warp per row, q read from global, same FP64 arithmetic.
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
  return warp_sum(acc);
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
    if ((threadIdx.x & 31) == 0) keys[qi * ld + doc] = desc_key((float)(dot * (double)inv_norm));
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
    if ((threadIdx.x & 31) == 0) keys[i] = desc_key((float)(dot * (double)inv_norm));
  }
}

// ---- table form ----------------------------------------------------------------
// Per query, T[n][v] = sum_{i<G} q[nG+i] * (code_i(v) - c) in FP64 for every
// 4-bit group n of a code row (G = 4 / BITS codes, MSB-first, c = (2^B-1)/2)
// and every nibble value v; a row's score is inv_norm * sum_n T[n][nib_n(row)].
// Each entry is a sum of G exact products (q * (code - c) needs at most 27
// significant bits), so the result agrees with the direct FP64 sum to ~1e-15.
// Lanes take rows (32 rows per warp) and walk the nibbles in step: a warp's
// shared-memory read stays inside one 128-byte group of 16 entries (at most 16
// distinct addresses, one wavefront), and each lane ends with its own row's
// sum, so no shuffles are needed.  Rows must be whole 16-byte chunks
// (dim * BITS % 128 == 0); the table (dim * BITS * 32 bytes) sits at a
// 4096-byte-aligned shared address so a group's address is base | offset.
constexpr int kTabThreads = 256;
constexpr uint32_t kTabMaxBytes = 200 * 1024;

__device__ __forceinline__ double lds_f64(uint32_t addr) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr));
  return v;
}

template <int BITS, bool SUBSET>
__global__ void __launch_bounds__(kTabThreads)
    asym_table_kernel(const uint8_t* __restrict__ codes, uint64_t n, uint32_t dim,
                      const float* __restrict__ q_unit, const uint64_t* __restrict__ off,
                      const uint32_t* __restrict__ cands, float inv_norm, uint32_t* __restrict__ keys,
                      uint64_t ld) {
  constexpr int G = 4 / BITS;
  constexpr uint32_t MASK = (1u << BITS) - 1;
  constexpr double C = ((double)(1u << BITS) - 1.0) * 0.5;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t t_base = ((uint32_t)__cvta_generic_to_shared(smem_raw) + 4095u) & ~4095u;
  double* T = reinterpret_cast<double*>(smem_raw + (t_base - (uint32_t)__cvta_generic_to_shared(smem_raw)));
  const uint64_t qi = blockIdx.y;
  const float* q = q_unit + qi * dim;
  const uint32_t n_nib = dim * BITS / 4;
  for (uint32_t e = threadIdx.x; e < n_nib * 16; e += kTabThreads) {
    const uint32_t g = e >> 4, v = e & 15;
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < G; i++) {
      const uint32_t code = (v >> (BITS * (G - 1 - i))) & MASK;
      acc += (double)q[g * G + i] * ((double)code - C);
    }
    T[e] = acc;
  }
  __syncthreads();

  uint64_t start, end;
  if (SUBSET) {
    start = off[qi];
    end = off[qi + 1];
  } else {
    start = 0;
    end = n;
  }
  const uint32_t bpv = dim * BITS / 8, chunks = bpv / 16;
  const int lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * kTabThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kTabThreads / 32;
  for (uint64_t base = start + gw * 32; base < end; base += nw * 32) {
    const uint64_t i = base + lane;
    const bool valid = i < end;
    const uint64_t row = valid ? (SUBSET ? (uint64_t)cands[i] : i) : 0;
    const uint4* rp = reinterpret_cast<const uint4*>(codes + row * bpv);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    uint4 x = valid ? __ldg(rp) : make_uint4(0, 0, 0, 0);
    for (uint32_t c = 0; c < chunks; c++) {
      const uint4 cur = x;
      if (c + 1 < chunks) x = valid ? __ldg(rp + c + 1) : make_uint4(0, 0, 0, 0);
      const uint32_t tb = t_base + c * 4096;  // 32 groups x 128 bytes
      const uint32_t w[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
      for (int k = 0; k < 4; k++) {
#pragma unroll
        for (int b = 0; b < 4; b++) {
#pragma unroll
          for (int h = 0; h < 2; h++) {  // high nibble first (MSB-first codes)
            const int sh = 8 * b + (h ? 0 : 4);
            const uint32_t o = sh >= 3 ? (w[k] >> (sh - 3)) & 0x78u : (w[k] << 3) & 0x78u;  // 8 * nibble
            const int nl = 8 * k + 2 * b + h;
            acc[nl & 3] += lds_f64((tb | o) + nl * 128);
          }
        }
      }
    }
    if (valid) {
      const float sc = (float)(((acc[0] + acc[1]) + (acc[2] + acc[3])) * (double)inv_norm);
      if (SUBSET)
        keys[i] = desc_key(sc);
      else
        keys[qi * ld + i] = desc_key(sc);
    }
  }
}

size_t table_smem(uint32_t dim, uint32_t bits) { return (size_t)dim * bits * 32 + 4096; }

bool table_ok(uint32_t dim, uint32_t bits) {
  const char* e = getenv("OVB_ASYM_TABLE");
  if (e && e[0] == '0') return false;
  return (uint64_t)dim * bits % 128 == 0 && (uint64_t)dim * bits * 32 <= kTabMaxBytes;
}

template <bool SUBSET>
void launch_table(uint32_t bits, dim3 grid, size_t smem, cudaStream_t st, const uint8_t* codes, uint64_t n,
                  uint32_t dim, const float* qu, const uint64_t* off, const uint32_t* cands, float inv_norm,
                  uint32_t* keys, uint64_t ld) {
#define OVB_TAB(B)                                                                                     \
  do {                                                                                                 \
    allow_dynamic_smem(asym_table_kernel<B, SUBSET>);                                                  \
    asym_table_kernel<B, SUBSET><<<grid, kTabThreads, smem, st>>>(codes, n, dim, qu, off, cands, inv_norm, \
                                                                  keys, ld);                           \
  } while (0)
  if (bits == 1)
    OVB_TAB(1);
  else if (bits == 2)
    OVB_TAB(2);
  else
    OVB_TAB(4);
#undef OVB_TAB
}

unsigned grid_x(uint64_t rows_per_cta, uint64_t n) {
  uint64_t g = (n + rows_per_cta - 1) / rows_per_cta;
  if (g < 1) g = 1;
  if (g > 148 * 8) g = 148 * 8;
  return (unsigned)g;
}

// Register path: rows are whole u32 words and a lane holds at most 32 query
// coordinates (dim <= 1024 for every bit width); W words per lane.
int plan_w(uint32_t dim, uint32_t bits) {
  if ((dim * bits) % 32 != 0) return 0;
  const uint32_t words = dim * bits / 32;
  const uint32_t W = (words + 31) / 32;
  if (W * (32 / bits) > 32) return 0;
  return W <= 1 ? 1 : W <= 2 ? 2 : 4;
}

template <int BITS>
void dispatch_bits(int W, bool subset, dim3 grid, cudaStream_t st, const uint8_t* codes, uint64_t n,
                   uint32_t dim, const float* qu, float inv_norm, uint32_t* keys, uint64_t ld,
                   const uint64_t* off, const uint32_t* cands) {
#define OVB_ASYM_CASE(WV)                                                                                  \
  if (W == WV) {                                                                                           \
    if (subset)                                                                                            \
      asym_subset_kernel<BITS, WV><<<grid, kThreads, 0, st>>>(codes, dim, qu, off, cands, inv_norm, keys); \
    else                                                                                                   \
      asym_scan_kernel<BITS, WV><<<grid, kThreads, 0, st>>>(codes, n, dim, qu, inv_norm, keys, ld);        \
    return;                                                                                                \
  }
  if constexpr (BITS == 1) {
    OVB_ASYM_CASE(1)
  } else if constexpr (BITS == 2) {
    OVB_ASYM_CASE(1)
    OVB_ASYM_CASE(2)
  } else {
    OVB_ASYM_CASE(1)
    OVB_ASYM_CASE(2)
    OVB_ASYM_CASE(4)
  }
#undef OVB_ASYM_CASE
}

void dispatch(uint32_t bits, int W, bool subset, dim3 grid, cudaStream_t st, const uint8_t* codes,
              uint64_t n, uint32_t dim, const float* qu, float inv_norm, uint32_t* keys, uint64_t ld,
              const uint64_t* off, const uint32_t* cands) {
  if (bits == 1)
    dispatch_bits<1>(W, subset, grid, st, codes, n, dim, qu, inv_norm, keys, ld, off, cands);
  else if (bits == 2)
    dispatch_bits<2>(W, subset, grid, st, codes, n, dim, qu, inv_norm, keys, ld, off, cands);
  else
    dispatch_bits<4>(W, subset, grid, st, codes, n, dim, qu, inv_norm, keys, ld, off, cands);
}

}  // namespace

void launch_asym_scan(const uint8_t* codes, uint64_t n, uint32_t dim, uint32_t bits,
                      const float* q_unit, uint64_t nq, float inv_norm, uint32_t* keys,
                      uint64_t ld, cudaStream_t stream) {
  if (!n || !nq) return;
  if (table_ok(dim, bits)) {
    // ~1024 rows per CTA: the table build stays a few percent of the scoring
    for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
      unsigned gy = (unsigned)((nq - q0) < 65535 ? (nq - q0) : 65535);
      dim3 grid(grid_x(1024, n), gy);
      launch_table<false>(bits, grid, table_smem(dim, bits), stream, codes, n, dim, q_unit + q0 * dim, nullptr,
                          nullptr, inv_norm, keys + q0 * ld, ld);
      launched();
    }
    return;
  }
  const int W = plan_w(dim, bits);
  for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
    unsigned gy = (unsigned)((nq - q0) < 65535 ? (nq - q0) : 65535);
    dim3 grid(grid_x(kThreads / 32, n), gy);
    if (W)
      dispatch(bits, W, false, grid, stream, codes, n, dim, q_unit + q0 * dim, inv_norm, keys + q0 * ld, ld,
               nullptr, nullptr);
    else
      asym_scan_generic<<<grid, kThreads, 0, stream>>>(codes, n, dim, bits, q_unit + q0 * dim, inv_norm,
                                                       keys + q0 * ld, ld);
    launched();
  }
}

void launch_asym_subset(const uint8_t* codes, uint32_t dim, uint32_t bits, const float* q_unit,
                        uint64_t nq, const uint64_t* offsets, const uint32_t* cands,
                        uint64_t max_row, float inv_norm, uint32_t* keys, cudaStream_t stream) {
  if (!nq || !max_row) return;
  // one arithmetic for every batch size, so a query scores the same alone and
  // inside a batch
  if (table_ok(dim, bits)) {
    // 512 rows per CTA (two per lane) with many queries, fewer with few
    const uint64_t rows_per_cta = nq >= 64 ? 512 : 128;
    for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
      unsigned gy = (unsigned)((nq - q0) < 65535 ? (nq - q0) : 65535);
      dim3 grid(grid_x(rows_per_cta, max_row), gy);
      launch_table<true>(bits, grid, table_smem(dim, bits), stream, codes, 0, dim, q_unit + q0 * dim,
                         offsets + q0, cands, inv_norm, keys, 0);
      launched();
    }
    return;
  }
  const int W = plan_w(dim, bits);
  // each warp loads its query slice once, so give it ~32 rows when there are
  // many queries; a single query spreads its rows over more CTAs
  const uint64_t rows_per_warp = nq >= 64 ? 32 : 4;
  for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
    unsigned gy = (unsigned)((nq - q0) < 65535 ? (nq - q0) : 65535);
    dim3 grid(grid_x((kThreads / 32) * rows_per_warp, max_row), gy);
    if (W)
      dispatch(bits, W, true, grid, stream, codes, 0, dim, q_unit + q0 * dim, inv_norm, keys, 0, offsets + q0,
               cands);
    else
      asym_subset_generic<<<grid, kThreads, 0, stream>>>(codes, dim, bits, q_unit + q0 * dim, offsets + q0,
                                                         cands, inv_norm, keys);
    launched();
  }
}

}  // namespace ovb
