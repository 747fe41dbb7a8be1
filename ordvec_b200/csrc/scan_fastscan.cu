// K3: FastScan b=2 nibble-LUT scorer (src/fastscan.rs:184-347).
//
// Per query the reference quantises one 16-entry u8 LUT per coordinate pair
// (built bit-exactly by fastscan_lut_kernel in prep.cu) and scores
//   acc  = sum_p lut[p][nibble_p(doc)]                      (exact u32)
//   score = (bias_sum + (acc as f32) * inv_q) * inv_norm     (fixed f32 ops)
// so integer accumulation plus the same three rounded f32 operations give
// scores -- and therefore candidate ids and tie order -- identical to the
// reference bit for bit.
//
// Device layout (B200-native, built at add/load time): the reference stores
// one nibble per byte at [block][pair][lane32].  Here two pairs share a byte,
// halving HBM traffic, and each lane's 32 pairs are contiguous:
//   [block][g = pair/32][lane 0..31][16 bytes], byte b = nib(32g+2b) | nib(32g+2b+1) << 4
// Pairs are padded to a multiple of 32 with LUT rows of zeros.  A warp owns a
// 32-document block; one coalesced 512-byte load per 32 pairs feeds 32
// shared-memory LUT lookups per lane.  QT queries share each loaded block.
#include "ovb_common.cuh"
#include "ovb_kernels.h"

namespace ovb {

namespace {

constexpr int kThreads = 256;

template <int QT>
__global__ void __launch_bounds__(kThreads)
    fastscan_scan_kernel(const uint8_t* __restrict__ blocks, uint64_t n, uint32_t pairs_pad,
                         const uint8_t* __restrict__ lut, const float* __restrict__ bias,
                         const float* __restrict__ invq, float inv_norm, uint64_t nq,
                         uint32_t* __restrict__ keys, uint64_t ld) {
  extern __shared__ __align__(16) uint8_t slut[];
  const uint64_t q0 = (uint64_t)blockIdx.y * QT;
  const int nqt = (int)((nq - q0) < (uint64_t)QT ? (nq - q0) : (uint64_t)QT);
  const uint32_t lut_bytes = pairs_pad * 16;
  {
    const uint4* src = (const uint4*)(lut + q0 * lut_bytes);
    uint4* dst = (uint4*)slut;
    const uint32_t n16 = (uint32_t)nqt * lut_bytes / 16;
    for (uint32_t i = threadIdx.x; i < n16; i += kThreads) dst[i] = src[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint32_t G = pairs_pad / 32;
  const uint64_t n_blocks = (n + 31) / 32;
  const uint64_t gw = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / 32;
  const uint64_t nw = (uint64_t)gridDim.x * kThreads / 32;
  for (uint64_t blk = gw; blk < n_blocks; blk += nw) {
    uint32_t acc[QT];
#pragma unroll
    for (int q = 0; q < QT; q++) acc[q] = 0;
    const uint4* src = (const uint4*)(blocks + blk * (uint64_t)lut_bytes) + lane;
    // four 16-byte code loads in flight per lane: a warp usually scores one
    // block, so one load at a time would leave it waiting on memory latency
    for (uint32_t g0 = 0; g0 < G; g0 += 4) {
      uint4 cv[4];
#pragma unroll
      for (int u = 0; u < 4; u++) cv[u] = g0 + u < G ? __ldcs(src + (g0 + u) * 32) : make_uint4(0, 0, 0, 0);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        if (g0 + u >= G) break;
        const uint32_t cw[4] = {cv[u].x, cv[u].y, cv[u].z, cv[u].w};
        const uint8_t* L = slut + (g0 + u) * 32 * 16;
#pragma unroll
        for (int q = 0; q < QT; q++) {
          const uint8_t* Lq = L + q * lut_bytes;
          uint32_t a = 0;
#pragma unroll
          for (int b = 0; b < 16; b++) {
            const uint32_t byte = (cw[b >> 2] >> (8 * (b & 3))) & 0xFF;
            a += Lq[(2 * b) * 16 + (byte & 15)];
            a += Lq[(2 * b + 1) * 16 + (byte >> 4)];
          }
          acc[q] += a;
        }
      }
    }
    const uint64_t doc = blk * 32 + lane;
    if (doc < n) {
#pragma unroll
      for (int q = 0; q < QT; q++) {
        if (q < nqt) {
          const float t = __fmul_rn(__uint2float_rn(acc[q]), invq[q0 + q]);
          const float raw = __fadd_rn(bias[q0 + q], t);
          keys[(q0 + q) * ld + doc] = desc_key(__fmul_rn(raw, inv_norm));
        }
      }
    }
  }
}

// reference layout [block][pair][lane] (one nibble per byte) -> device layout
__global__ void fastscan_relayout_kernel(const uint8_t* __restrict__ ref, uint64_t n,
                                         uint32_t pairs, uint32_t pairs_pad,
                                         uint8_t* __restrict__ dev) {
  const uint64_t n_blocks = (n + 31) / 32;
  const uint64_t total = n_blocks * (pairs_pad / 2) * 32;  // output bytes
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t blk = t / ((uint64_t)(pairs_pad / 2) * 32);
    const uint32_t r = (uint32_t)(t % ((uint64_t)(pairs_pad / 2) * 32));
    const uint32_t g = r / 512, lane = (r % 512) / 16, b = r % 16;
    const uint32_t p0 = g * 32 + 2 * b, p1 = p0 + 1;
    const uint64_t rb = blk * (uint64_t)pairs * 32;
    uint8_t lo = p0 < pairs ? (ref[rb + (uint64_t)p0 * 32 + lane] & 15) : 0;
    uint8_t hi = p1 < pairs ? (ref[rb + (uint64_t)p1 * 32 + lane] & 15) : 0;
    dev[t] = (uint8_t)(lo | (hi << 4));
  }
}

}  // namespace

uint32_t fastscan_pairs_pad(uint32_t dim) { return ((dim / 2 + 31) / 32) * 32; }
uint64_t fastscan_block_bytes(uint32_t pairs_pad) { return (uint64_t)pairs_pad * 16; }

void launch_fastscan_scan(const uint8_t* blocks, uint64_t n, uint32_t pairs_pad,
                          const uint8_t* lut, const float* bias_sum, const float* inv_q,
                          float inv_norm, uint64_t nq, uint32_t* keys, uint64_t ld,
                          cudaStream_t stream) {
  if (!n || !nq) return;
  const uint64_t n_blocks = (n + 31) / 32;
  if ((size_t)pairs_pad * 16 > 227 * 1024)
    throw std::invalid_argument("FastScan dim too large for the shared-memory LUT (dim <= 16384)");
  int qt = nq >= 8 ? 8 : nq >= 4 ? 4 : nq >= 2 ? 2 : 1;
  while (qt > 1 && (size_t)qt * pairs_pad * 16 > 227 * 1024) qt >>= 1;
  const size_t smem1 = (size_t)qt * pairs_pad * 16;
  uint64_t gx = (n_blocks + (kThreads / 32) - 1) / (kThreads / 32);
  if (gx > 148 * 8) gx = 148 * 8;
  for (uint64_t q0 = 0; q0 < nq; q0 += (uint64_t)qt * 65535) {
    uint64_t rem = nq - q0;
    unsigned gy = (unsigned)(((rem + qt - 1) / qt) < 65535 ? ((rem + qt - 1) / qt) : 65535);
    dim3 grid((unsigned)gx, gy);
    const uint8_t* l = lut + q0 * pairs_pad * 16;
#define OVB_FS(QTV)                                                                                   \
  case QTV:                                                                                           \
    allow_dynamic_smem(fastscan_scan_kernel<QTV>);                                                    \
    fastscan_scan_kernel<QTV><<<grid, kThreads, smem1, stream>>>(blocks, n, pairs_pad, l, bias_sum + q0,   \
                                                                 inv_q + q0, inv_norm, rem, keys + q0 * ld, ld); \
    break;
    switch (qt) {
      OVB_FS(1)
      OVB_FS(2)
      OVB_FS(4)
      OVB_FS(8)
    }
#undef OVB_FS
    launched();
  }
}

void launch_fastscan_relayout(const uint8_t* ref_blocks, uint64_t n, uint32_t pairs,
                              uint32_t pairs_pad, uint8_t* dev_blocks, cudaStream_t stream) {
  if (!n) return;
  fastscan_relayout_kernel<<<148 * 8, 256, 0, stream>>>(ref_blocks, n, pairs, pairs_pad, dev_blocks);
  launched();
}

}  // namespace ovb
