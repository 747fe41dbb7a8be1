// K1 / K2 / K6: popcount scans over sign bitmaps, constant-weight bitmaps and
// multi-bucket bitmaps.
//
// * sign   (src/sign_bitmap.rs:674-753)  key32 = popcount(q XOR d)   (Hamming)
// * bitmap (src/bitmap.rs:607-679)       key32 = n_top - popcount(q AND d)
// * multi-bucket (src/multi_bucket.rs:194-222)  f32 sum over (a, b) of
//   W[a,b] * popcount(Q_a AND D_b) in (a, b) order, key32 = desc_key(score).
//
// Layout: rows of `qpv` u64 words (bit j of word j/64, LSB first), exactly the
// reference's in-memory/on-disk layout.  A group of LPD lanes (a power of two
// covering the row's words) reads one row, so a warp instruction touches
// 32/LPD consecutive rows = one contiguous span of HBM; partial popcounts are
// summed with xor-shuffles inside the group.  Query words stay in registers.
// Integer results are exact, so every path is bit-identical to the reference.
#include "ovb_common.cuh"
#include "ovb_kernels.h"

namespace ovb {

namespace {

constexpr int kThreads = 256;

template <int LPD, int WPL>
__global__ void __launch_bounds__(kThreads)
    popc_scan_kernel(int mode, const uint64_t* __restrict__ words, uint64_t n, uint32_t qpv,
                     const uint64_t* __restrict__ qbits, uint32_t n_top,
                     uint32_t* __restrict__ keys, uint64_t ld) {
  constexpr int DPW = 32 / LPD;
  const uint64_t qi = blockIdx.y;
  const uint64_t* qb = qbits + qi * qpv;
  const int lane = threadIdx.x & 31;
  const int g = lane % LPD;
  uint64_t qreg[WPL];
#pragma unroll
  for (int i = 0; i < WPL; i++) {
    uint32_t w = g + i * LPD;
    qreg[i] = w < qpv ? qb[w] : 0;
  }
  const uint64_t gw = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kThreads / 32;
  uint32_t* out = keys + qi * ld;
  for (uint64_t base = gw * DPW; base < n; base += nw * DPW) {
    const uint64_t doc = base + lane / LPD;
    uint32_t acc = 0;
    if (doc < n) {
      const uint64_t* d = words + doc * qpv;
#pragma unroll
      for (int i = 0; i < WPL; i++) {
        uint32_t w = g + i * LPD;
        if (w < qpv) {
          uint64_t x = __ldcs((const unsigned long long*)(d + w));
          acc += __popcll(mode == 0 ? (x ^ qreg[i]) : (x & qreg[i]));
        }
      }
    }
#pragma unroll
    for (int o = LPD / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if (g == 0 && doc < n) out[doc] = mode == 0 ? acc : n_top - acc;
  }
}

// Generic fallback for rows wider than 4 words per lane (dim > 8192).
__global__ void __launch_bounds__(kThreads)
    popc_scan_wide_kernel(int mode, const uint64_t* __restrict__ words, uint64_t n,
                          uint32_t qpv, const uint64_t* __restrict__ qbits, uint32_t n_top,
                          uint32_t* __restrict__ keys, uint64_t ld) {
  const uint64_t qi = blockIdx.y;
  const uint64_t* qb = qbits + qi * qpv;
  const int lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kThreads / 32;
  for (uint64_t doc = gw; doc < n; doc += nw) {
    const uint64_t* d = words + doc * qpv;
    uint32_t acc = 0;
    for (uint32_t w = lane; w < qpv; w += 32) {
      uint64_t x = d[w];
      acc += __popcll(mode == 0 ? (x ^ qb[w]) : (x & qb[w]));
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if (lane == 0) keys[qi * ld + doc] = mode == 0 ? acc : n_top - acc;
  }
}

__global__ void __launch_bounds__(kThreads)
    popc_subset_kernel(int mode, const uint64_t* __restrict__ words, uint32_t qpv,
                       const uint64_t* __restrict__ qbits, const uint64_t* __restrict__ off,
                       const uint32_t* __restrict__ cands, uint32_t n_top,
                       uint32_t* __restrict__ keys) {
  const uint64_t qi = blockIdx.y;
  const uint64_t s = off[qi], e = off[qi + 1];
  const uint64_t* qb = qbits + qi * qpv;
  const int lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kThreads / 32;
  for (uint64_t i = s + gw; i < e; i += nw) {
    const uint64_t* d = words + (uint64_t)cands[i] * qpv;
    uint32_t acc = 0;
    for (uint32_t w = lane; w < qpv; w += 32) {
      uint64_t x = d[w];
      acc += __popcll(mode == 0 ? (x ^ qb[w]) : (x & qb[w]));
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if (lane == 0) keys[i] = mode == 0 ? acc : n_top - acc;
  }
}

// One warp per document; lanes stride the words of each bucket bitmap.
__global__ void __launch_bounds__(kThreads)
    multibucket_scan_kernel(const uint64_t* __restrict__ words, uint64_t n, uint32_t qpb,
                            uint32_t nb, const uint64_t* __restrict__ qbits,
                            const float* __restrict__ wts, uint32_t* __restrict__ keys,
                            uint64_t ld) {
  __shared__ float sw[256];
  const uint64_t qi = blockIdx.y;
  for (uint32_t i = threadIdx.x; i < nb * nb; i += blockDim.x) sw[i] = wts[i];
  __syncthreads();
  const uint64_t* qb = qbits + qi * (uint64_t)nb * qpb;
  const int lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kThreads / 32;
  const uint64_t per_doc = (uint64_t)nb * qpb;
  for (uint64_t doc = gw; doc < n; doc += nw) {
    const uint64_t* d = words + doc * per_doc;
    float acc = 0.0f;
    for (uint32_t a = 0; a < nb; a++)
      for (uint32_t b = 0; b < nb; b++) {
        const float wt = sw[a * nb + b];
        if (wt == 0.0f) continue;
        uint32_t ov = 0;
        for (uint32_t w = lane; w < qpb; w += 32) ov += __popcll(qb[a * qpb + w] & d[b * qpb + w]);
        for (int o = 16; o > 0; o >>= 1) ov += __shfl_xor_sync(0xFFFFFFFFu, ov, o);
        acc = __fadd_rn(acc, __fmul_rn(wt, (float)ov));
      }
    if (lane == 0) keys[qi * ld + doc] = desc_key(acc);
  }
}

unsigned scan_grid(uint64_t units_per_cta, uint64_t n) {
  uint64_t g = (n + units_per_cta - 1) / units_per_cta;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (unsigned)g;
}

template <int LPD>
void launch_lpd(int mode, const uint64_t* words, uint64_t n, uint32_t qpv, const uint64_t* qbits,
                unsigned gy, uint32_t n_top, uint32_t* keys, uint64_t ld, cudaStream_t stream) {
  dim3 grid(scan_grid((kThreads / 32) * (32 / LPD), n), gy);
  uint32_t wpl = (qpv + LPD - 1) / LPD;
  if (wpl <= 1)
    popc_scan_kernel<LPD, 1><<<grid, kThreads, 0, stream>>>(mode, words, n, qpv, qbits, n_top, keys, ld);
  else if (wpl == 2)
    popc_scan_kernel<LPD, 2><<<grid, kThreads, 0, stream>>>(mode, words, n, qpv, qbits, n_top, keys, ld);
  else
    popc_scan_kernel<LPD, 4><<<grid, kThreads, 0, stream>>>(mode, words, n, qpv, qbits, n_top, keys, ld);
}

}  // namespace

void launch_popc_scan(int mode, const uint64_t* words, uint64_t n, uint32_t qpv,
                      const uint64_t* qbits, uint64_t nq, uint32_t n_top, uint32_t* keys,
                      uint64_t ld, cudaStream_t stream) {
  if (!n || !nq) return;
  for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
    unsigned gy = (unsigned)((nq - q0) < 65535 ? (nq - q0) : 65535);
    const uint64_t* qb = qbits + q0 * qpv;
    uint32_t* kk = keys + q0 * ld;
    if (qpv > 128) {
      dim3 grid(scan_grid(kThreads / 32, n), gy);
      popc_scan_wide_kernel<<<grid, kThreads, 0, stream>>>(mode, words, n, qpv, qb, n_top, kk, ld);
    } else if (qpv <= 1) {
      launch_lpd<1>(mode, words, n, qpv, qb, gy, n_top, kk, ld, stream);
    } else if (qpv <= 2) {
      launch_lpd<2>(mode, words, n, qpv, qb, gy, n_top, kk, ld, stream);
    } else if (qpv <= 4) {
      launch_lpd<4>(mode, words, n, qpv, qb, gy, n_top, kk, ld, stream);
    } else if (qpv <= 8) {
      launch_lpd<8>(mode, words, n, qpv, qb, gy, n_top, kk, ld, stream);
    } else if (qpv <= 16) {
      launch_lpd<16>(mode, words, n, qpv, qb, gy, n_top, kk, ld, stream);
    } else {
      launch_lpd<32>(mode, words, n, qpv, qb, gy, n_top, kk, ld, stream);
    }
    launched();
  }
}

void launch_popc_subset(int mode, const uint64_t* words, uint32_t qpv, const uint64_t* qbits,
                        uint64_t nq, const uint64_t* offsets, const uint32_t* cands,
                        uint64_t max_row, uint32_t n_top, uint32_t* keys, cudaStream_t stream) {
  if (!nq || !max_row) return;
  for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
    unsigned gy = (unsigned)((nq - q0) < 65535 ? (nq - q0) : 65535);
    dim3 grid(scan_grid(kThreads / 32, max_row), gy);
    popc_subset_kernel<<<grid, kThreads, 0, stream>>>(mode, words, qpv, qbits + q0 * qpv, offsets + q0,
                                                      cands, n_top, keys);
    launched();
  }
}

void launch_multibucket_scan(const uint64_t* words, uint64_t n, uint32_t qpb, uint32_t nb,
                             const uint64_t* qbits, const float* w, uint64_t nq, uint32_t* keys,
                             uint64_t ld, cudaStream_t stream) {
  if (!n || !nq) return;
  for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
    unsigned gy = (unsigned)((nq - q0) < 65535 ? (nq - q0) : 65535);
    dim3 grid(scan_grid(kThreads / 32, n), gy);
    multibucket_scan_kernel<<<grid, kThreads, 0, stream>>>(words, n, qpb, nb, qbits + q0 * (uint64_t)nb * qpb,
                                                           w, keys + q0 * ld, ld);
    launched();
  }
}

}  // namespace ovb
