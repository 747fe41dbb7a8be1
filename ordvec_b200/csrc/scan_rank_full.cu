// K9: the full-precision Rank index (u16 rank per coordinate, src/rank.rs:283-482).
//
// * symmetric (Rank::search, src/rank.rs:364-419): Spearman in exact integers,
//   acc = sum_d (2 q_r[d] - (D - 1)) (2 d_r[d] - (D - 1)) in i64, then
//   score = ((acc as f32) * 0.25) * (1 / norm^2) in f32, left to right.  A warp
//   per document reads its row with 16-byte loads (8 ranks per lane per step,
//   coalesced) against the query's centred ranks in shared memory; the i64
//   partial sums meet in a warp reduction.  Integer sums are order-free, so
//   the score is the reference's bit for bit.
// * asymmetric (Rank::search_asymmetric, src/rank.rs:420-482):
//   acc = sequential f32 sum over d of q_unit[d] * (rank as f32), then
//   score = (acc - mean * q_sum) * (1 / norm).  The reference's sum is a
//   dependent chain in coordinate order, so each lane owns one document and
//   runs that chain (round-to-nearest, no contraction); the query lives in
//   shared memory (one address for all lanes: broadcast).
#include <cmath>

#include "ovb_common.cuh"
#include "ovb_kernels.h"

namespace ovb {

namespace {

constexpr int kRfThreads = 256;

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
  const bool vec = dim % 8 == 0;  // rows start 16-byte aligned
  for (uint64_t doc = gw; doc < n; doc += nw) {
    const uint16_t* row = ranks + doc * dim;
    long long acc = 0;
    if (vec) {
      for (uint32_t j0 = 8 * lane; j0 < dim; j0 += 256) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(row + j0));
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
          acc += (long long)qc[j0 + 2 * i] * (2 * (int32_t)(w[i] & 0xFFFF) - m2);
          acc += (long long)qc[j0 + 2 * i + 1] * (2 * (int32_t)(w[i] >> 16) - m2);
        }
      }
    } else {
      for (uint32_t j = lane; j < dim; j += 32) acc += (long long)qc[j] * (2 * (int32_t)__ldg(row + j) - m2);
    }
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
    if (dim % 8 == 0) {
      for (uint32_t j0 = 0; j0 < dim; j0 += 8) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(row + j0));
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
          acc = __fadd_rn(acc, __fmul_rn(qs[j0 + 2 * i], (float)(w[i] & 0xFFFF)));
          acc = __fadd_rn(acc, __fmul_rn(qs[j0 + 2 * i + 1], (float)(w[i] >> 16)));
        }
      }
    } else {
      for (uint32_t j = 0; j < dim; j++) acc = __fadd_rn(acc, __fmul_rn(qs[j], (float)__ldg(row + j)));
    }
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
  const size_t smem = (size_t)dim * 4;
  if (smem > 48 * 1024)
    OVB_CUDA(cudaFuncSetAttribute(rank_sym_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
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
  const size_t smem = (size_t)dim * 4;
  if (smem > 48 * 1024)
    OVB_CUDA(cudaFuncSetAttribute(rank_asym_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
    const unsigned gy = (unsigned)(nq - q0 < 65535 ? nq - q0 : 65535);
    rank_asym_kernel<<<dim3(rf_grid(n, kRfThreads), gy), kRfThreads, smem, stream>>>(
        ranks, n, dim, q_unit + q0 * dim, q_sum + q0, mean, inv_norm, keys + q0 * ld, ld);
    launched();
  }
}

}  // namespace ovb
