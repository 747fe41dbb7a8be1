// K9: the full-precision Rank index (u16 rank per coordinate, src/rank.rs:283-482).
//
// * symmetric (Rank::search, src/rank.rs:364-419): the reference sums
//   (2 q_r - (D - 1)) (2 d_r - (D - 1)) in i64 and scores
//   ((acc as f32) * 0.25) * (1 / norm^2) in f32, left to right.  Rows are
//   permutations of [0, D) (the encoder makes them so and the .ovr loader
//   checks it), so sum q_r = sum d_r = D (D - 1) / 2 and
//       acc = 4 sum_d q_r d_r - D (D - 1)^2,
//   the same integer, from a plain u32 dot product (sum q_r d_r <= sum r^2 <
//   2^32 for D <= 2048; u64 above).  The score is the reference's bit for bit.
// * asymmetric (Rank::search_asymmetric, src/rank.rs:420-482):
//   acc = sequential f32 sum over d of q_unit[d] * (rank as f32), then
//   score = (acc - mean * q_sum) * (1 / norm).  The sum is a dependent chain in
//   coordinate order, so each lane owns one document and runs that chain
//   (round-to-nearest, no contraction) for each of its queries.
//
// Staged, query-tiled form (dim a multiple of 8): a lane owns one document
// and QT queries.  A warp stages its 32 rows through shared memory in chunks
// of 32 coordinates (coalesced 16-byte loads, the next chunk's loads in flight
// while the current one is scored; rows padded to 17 words so the lanes' reads
// hit distinct banks) and reads the QT queries' values for a coordinate as one
// broadcast.  A row crosses HBM once per QT queries; the grid's x is the query
// group, so the groups sharing a document chunk run side by side and share it
// through L2.  Other dims take a warp-per-document (symmetric) or
// lane-per-document (asymmetric) form that reads rows with scalar loads.
#include <cmath>
#include <type_traits>

#include "ovb_common.cuh"
#include "ovb_kernels.h"

namespace ovb {

namespace {

constexpr int kRfThreads = 256;
constexpr int kRfWarps = kRfThreads / 32;
constexpr int kChunk = 32;                 // coordinates per staged chunk
constexpr int kRowWords = kChunk / 2 + 1;  // 16 rank pairs + 1 pad word

// SYM: q holds u16 ranks, staged as qv[j * QT + t] u32; !SYM: f32 unit-query values.
template <bool SYM, int QT, bool WIDE>
__global__ void __launch_bounds__(kRfThreads)
    rank_tile_kernel(const uint16_t* __restrict__ ranks, uint64_t n, uint32_t dim, const void* __restrict__ q,
                     const float* __restrict__ q_sum, uint64_t nq, float mean, float scale,
                     uint32_t* __restrict__ keys, uint64_t ld) {
  using Acc = typename std::conditional<WIDE, unsigned long long, uint32_t>::type;
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* rows = smem;                            // [warp][32][kRowWords]
  uint32_t* qv = smem + kRfWarps * 32 * kRowWords;  // [dim][QT]
  const uint64_t g0 = (uint64_t)blockIdx.x * QT;    // first query of the group
  for (uint32_t e = threadIdx.x; e < dim * QT; e += kRfThreads) {
    const uint32_t j = e / QT, t = e % QT;
    const uint64_t qi = g0 + t < nq ? g0 + t : nq - 1;  // padding queries repeat the last
    qv[e] = SYM ? (uint32_t)((const uint16_t*)q)[qi * dim + j] : __float_as_uint(((const float*)q)[qi * dim + j]);
  }
  __syncthreads();
  const int warp = threadIdx.x / 32, lane = threadIdx.x & 31;
  uint32_t* wrow = rows + warp * 32 * kRowWords;
  const uint32_t n_chunks = (dim + kChunk - 1) / kChunk;
  for (uint64_t d0 = ((uint64_t)blockIdx.y * kRfWarps + warp) * 32; d0 < n;
       d0 += (uint64_t)gridDim.y * kRfWarps * 32) {
    Acc dot[QT];
    float acc[QT];
#pragma unroll
    for (int t = 0; t < QT; t++) {
      dot[t] = 0;
      acc[t] = 0.0f;
    }
    // lane l loads 16-byte piece p = l % 4 of rows l / 4 + 8 i (i = 0..3)
    uint4 buf[4];
    auto load = [&](uint32_t c) {
      const uint32_t c0 = c * kChunk, pieces = (dim - c0 < (uint32_t)kChunk ? dim - c0 : kChunk) / 8;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const uint32_t r = (uint32_t)lane / 4 + 8 * i, p = (uint32_t)lane % 4;
        const uint64_t doc = d0 + r;
        buf[i] = (doc < n && p < pieces) ? __ldg(reinterpret_cast<const uint4*>(ranks + doc * dim + c0 + 8 * p))
                                         : make_uint4(0, 0, 0, 0);
      }
    };
    load(0);
    for (uint32_t c = 0; c < n_chunks; c++) {
      __syncwarp();
#pragma unroll
      for (int i = 0; i < 4; i++) {
        uint32_t* dst = wrow + ((uint32_t)lane / 4 + 8 * i) * kRowWords + ((uint32_t)lane % 4) * 4;
        dst[0] = buf[i].x;
        dst[1] = buf[i].y;
        dst[2] = buf[i].z;
        dst[3] = buf[i].w;
      }
      __syncwarp();
      if (c + 1 < n_chunks) load(c + 1);
      const uint32_t c0 = c * kChunk, words = (dim - c0 < (uint32_t)kChunk ? dim - c0 : kChunk) / 2;
      const uint32_t* my = wrow + lane * kRowWords;
      for (uint32_t w = 0; w < words; w++) {
        const uint32_t x = my[w];
        const uint32_t* q0 = qv + (c0 + 2 * w) * QT;
        const uint32_t* q1 = q0 + QT;
        if (SYM) {
          const uint32_t r0 = x & 0xFFFFu, r1 = x >> 16;
#pragma unroll
          for (int t = 0; t < QT; t++) dot[t] += (Acc)r0 * q0[t] + (Acc)r1 * q1[t];
        } else {
          const float f0 = __uint2float_rn(x & 0xFFFFu), f1 = __uint2float_rn(x >> 16);
#pragma unroll
          for (int t = 0; t < QT; t++) {
            acc[t] = __fadd_rn(acc[t], __fmul_rn(__uint_as_float(q0[t]), f0));
            acc[t] = __fadd_rn(acc[t], __fmul_rn(__uint_as_float(q1[t]), f1));
          }
        }
      }
    }
    const uint64_t doc = d0 + lane;
    if (doc < n) {
      const long long base = (long long)dim * (long long)(dim - 1) * (long long)(dim - 1);
#pragma unroll
      for (int t = 0; t < QT; t++) {
        const uint64_t qi = g0 + t;
        if (qi < nq) {
          float s;
          if (SYM) {
            const long long a = 4 * (long long)dot[t] - base;
            s = __fmul_rn(__fmul_rn(__ll2float_rn(a), 0.25f), scale);
          } else {
            s = __fmul_rn(__fsub_rn(acc[t], __fmul_rn(mean, q_sum[qi])), scale);
          }
          keys[qi * ld + doc] = desc_key(s);
        }
      }
    }
  }
}

// Scalar forms for dims that are not a multiple of 8 (rows not 16-byte aligned).
__global__ void __launch_bounds__(kRfThreads)
    rank_sym_kernel(const uint16_t* __restrict__ ranks, uint64_t n, uint32_t dim,
                    const uint16_t* __restrict__ q_ranks, float inv_norm_sq, uint32_t* __restrict__ keys,
                    uint64_t ld) {
  extern __shared__ int32_t qc[];  // 2 q_r - (D - 1)
  const uint64_t qi = blockIdx.y;
  const int32_t m2 = (int32_t)dim - 1;
  for (uint32_t j = threadIdx.x; j < dim; j += blockDim.x) qc[j] = 2 * (int32_t)q_ranks[qi * dim + j] - m2;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * kRfThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kRfThreads / 32;
  for (uint64_t doc = gw; doc < n; doc += nw) {
    const uint16_t* row = ranks + doc * dim;
    long long acc = 0;
    for (uint32_t j = lane; j < dim; j += 32) acc += (long long)qc[j] * (2 * (int32_t)__ldg(row + j) - m2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if (lane == 0) keys[qi * ld + doc] = desc_key(__fmul_rn(__fmul_rn(__ll2float_rn(acc), 0.25f), inv_norm_sq));
  }
}

__global__ void __launch_bounds__(kRfThreads)
    rank_asym_kernel(const uint16_t* __restrict__ ranks, uint64_t n, uint32_t dim,
                     const float* __restrict__ q_unit, const float* __restrict__ q_sum, float mean,
                     float inv_norm, uint32_t* __restrict__ keys, uint64_t ld) {
  extern __shared__ float qs[];
  const uint64_t qi = blockIdx.y;
  for (uint32_t j = threadIdx.x; j < dim; j += blockDim.x) qs[j] = q_unit[qi * dim + j];
  __syncthreads();
  const float shift = __fmul_rn(mean, q_sum[qi]);
  for (uint64_t doc = (uint64_t)blockIdx.x * kRfThreads + threadIdx.x; doc < n;
       doc += (uint64_t)gridDim.x * kRfThreads) {
    const uint16_t* row = ranks + doc * dim;
    float acc = 0.0f;
    for (uint32_t j = 0; j < dim; j++) acc = __fadd_rn(acc, __fmul_rn(qs[j], (float)__ldg(row + j)));
    keys[qi * ld + doc] = desc_key(__fmul_rn(__fsub_rn(acc, shift), inv_norm));
  }
}

// q_sum = sequential f32 sum of each q_unit row (Iterator::sum order)
__global__ void row_sum_kernel(const float* __restrict__ q, uint64_t nq, uint32_t dim, float* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  float s = -0.0f;
  for (uint32_t j = 0; j < dim; j++) s = __fadd_rn(s, q[i * dim + j]);
  out[i] = s;
}

unsigned rf_grid(uint64_t units, uint64_t per_cta) {
  uint64_t g = (units + per_cta - 1) / per_cta;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (unsigned)g;
}

// queries per tile: as many as the batch has, up to 8, while the query block
// stays within 64 KiB of shared memory
int rank_qt(uint64_t nq, uint32_t dim) {
  if (nq >= 8 && (uint64_t)dim * 8 * 4 <= 64 * 1024) return 8;
  if (nq >= 4 && (uint64_t)dim * 4 * 4 <= 64 * 1024) return 4;
  return 1;
}

template <bool SYM, int QT, bool WIDE>
void launch_tile(const uint16_t* ranks, uint64_t n, uint32_t dim, const void* q, const float* q_sum, uint64_t nq,
                 float mean, float scale, uint32_t* keys, uint64_t ld, cudaStream_t stream) {
  const size_t smem = ((size_t)kRfWarps * 32 * kRowWords + (size_t)dim * QT) * 4;
  auto kern = rank_tile_kernel<SYM, QT, WIDE>;
  allow_dynamic_smem(kern);
  const uint64_t groups = (nq + QT - 1) / QT;
  uint64_t gy = (n + kRfWarps * 32 - 1) / (kRfWarps * 32);
  // enough CTAs to fill every SM several times over; documents beyond that loop
  const uint64_t want = 148ull * 32;
  if (gy * groups > want) gy = (want + groups - 1) / groups;
  if (gy < 1) gy = 1;
  if (gy > 65535) gy = 65535;
  for (uint64_t g0 = 0; g0 < groups; g0 += 0x7FFFFFFF) {
    const uint64_t gn = groups - g0 < 0x7FFFFFFF ? groups - g0 : 0x7FFFFFFF;
    const uint64_t q0 = g0 * QT;
    const void* qp = SYM ? (const void*)((const uint16_t*)q + q0 * dim) : (const void*)((const float*)q + q0 * dim);
    kern<<<dim3((unsigned)gn, (unsigned)gy), kRfThreads, smem, stream>>>(
        ranks, n, dim, qp, q_sum ? q_sum + q0 : nullptr, nq - q0, mean, scale, keys + q0 * ld, ld);
    launched();
  }
}

template <bool SYM, bool WIDE>
void launch_tiled(int qt, const uint16_t* ranks, uint64_t n, uint32_t dim, const void* q, const float* q_sum,
                  uint64_t nq, float mean, float scale, uint32_t* keys, uint64_t ld, cudaStream_t stream) {
  if (qt == 8)
    launch_tile<SYM, 8, WIDE>(ranks, n, dim, q, q_sum, nq, mean, scale, keys, ld, stream);
  else if (qt == 4)
    launch_tile<SYM, 4, WIDE>(ranks, n, dim, q, q_sum, nq, mean, scale, keys, ld, stream);
  else
    launch_tile<SYM, 1, WIDE>(ranks, n, dim, q, q_sum, nq, mean, scale, keys, ld, stream);
}

}  // namespace

// rank_norm (src/rank.rs:249-252) in f32
float rank_norm_f32(uint32_t dim) {
  const double d = (double)dim;
  return (float)std::sqrt(d * (d * d - 1.0) / 12.0);
}

void launch_rank_sym_scan(const uint16_t* ranks, uint64_t n, uint32_t dim, const uint16_t* q_ranks, uint64_t nq,
                          uint32_t* keys, uint64_t ld, cudaStream_t stream) {
  if (!n || !nq) return;
  const float norm = rank_norm_f32(dim);
  const float inv_norm_sq = 1.0f / (norm * norm);
  if (dim % 8 == 0) {
    const int qt = rank_qt(nq, dim);
    if (dim <= 2048)
      launch_tiled<true, false>(qt, ranks, n, dim, q_ranks, nullptr, nq, 0.0f, inv_norm_sq, keys, ld, stream);
    else
      launch_tiled<true, true>(qt, ranks, n, dim, q_ranks, nullptr, nq, 0.0f, inv_norm_sq, keys, ld, stream);
    return;
  }
  const size_t smem = (size_t)dim * 4;
  allow_dynamic_smem(rank_sym_kernel);
  for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
    const unsigned gy = (unsigned)(nq - q0 < 65535 ? nq - q0 : 65535);
    rank_sym_kernel<<<dim3(rf_grid(n, kRfThreads / 32), gy), kRfThreads, smem, stream>>>(
        ranks, n, dim, q_ranks + q0 * dim, inv_norm_sq, keys + q0 * ld, ld);
    launched();
  }
}

void launch_rank_asym_scan(const uint16_t* ranks, uint64_t n, uint32_t dim, const float* q_unit, float* q_sum,
                           uint64_t nq, uint32_t* keys, uint64_t ld, cudaStream_t stream) {
  if (!n || !nq) return;
  row_sum_kernel<<<(unsigned)((nq + 127) / 128), 128, 0, stream>>>(q_unit, nq, dim, q_sum);
  launched();
  const float inv_norm = 1.0f / rank_norm_f32(dim);
  const float mean = ((float)dim - 1.0f) / 2.0f;
  if (dim % 8 == 0) {
    launch_tiled<false, false>(rank_qt(nq, dim), ranks, n, dim, q_unit, q_sum, nq, mean, inv_norm, keys, ld, stream);
    return;
  }
  const size_t smem = (size_t)dim * 4;
  allow_dynamic_smem(rank_asym_kernel);
  for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
    const unsigned gy = (unsigned)(nq - q0 < 65535 ? nq - q0 : 65535);
    rank_asym_kernel<<<dim3(rf_grid(n, kRfThreads), gy), kRfThreads, smem, stream>>>(
        ranks, n, dim, q_unit + q0 * dim, q_sum + q0, mean, inv_norm, keys + q0 * ld, ld);
    launched();
  }
}

}  // namespace ovb
