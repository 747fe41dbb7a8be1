// K1 / K2 / K6: popcount scans over sign bitmaps, constant-weight bitmaps and
// multi-bucket bitmaps.
//
// * sign   (src/sign_bitmap.rs:674-753)  key32 = popcount(q XOR d)   (Hamming)
// * bitmap (src/bitmap.rs:607-679)       key32 = n_top - popcount(q AND d)
// * multi-bucket (src/multi_bucket.rs:194-222)  f32 sum over (a, b) of
//   W[a,b] * popcount(Q_a AND D_b) in (a, b) order, key32 = desc_key(score).
//
// Layout: rows of `qpv` u64 words (bit j of word j/64, LSB first), exactly the
// reference's in-memory/on-disk layout.  Full scans run one lane per row with
// eight independent word loads in flight per lane (the stream is bound by
// bytes in flight); up to eight queries share each row read.  The subset form
// runs a warp per candidate.  Integer results are exact, so every path is
// bit-identical to the reference.
#include "ovb_common.cuh"
#include "ovb_kernels.h"

namespace ovb {

namespace {

constexpr int kThreads = 256;

// One lane per row.  The row's words are read 8 at a time (8 independent
// loads in flight per lane); the lanes of a warp read 32 consecutive rows, so
// the sectors a load instruction misses are the ones its successors hit in L1
// and every byte crosses HBM once.  Up to QG queries share each row read; their
// words sit in shared memory (same address in every lane: broadcast).
// Up to 8 words of a row starting at p (count of them valid, rest 0); with VEC
// (p 16-byte aligned, even count) as 16-byte loads, so a sector is consumed
// by back-to-back instructions.
template <bool VEC>
__device__ __forceinline__ void load_words8(const uint64_t* __restrict__ p, uint32_t count, uint64_t (&x)[8]) {
  if (VEC) {
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
      if ((uint32_t)i < count) {
        const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(p + i));
        x[i] = v.x;
        x[i + 1] = v.y;
      } else {
        x[i] = x[i + 1] = 0ull;
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < 8; i++) x[i] = (uint32_t)i < count ? __ldg(p + i) : 0ull;
  }
}

template <int QG, bool VEC>
__global__ void __launch_bounds__(kThreads)
    popc_rows_kernel(int mode, const uint64_t* __restrict__ words, uint64_t n, uint32_t qpv,
                     const uint64_t* __restrict__ qbits, uint64_t nq, uint32_t n_top,
                     uint32_t* __restrict__ keys, uint64_t ld) {
  extern __shared__ uint64_t sq[];  // QG x qpv query words
  const uint64_t q0 = (uint64_t)blockIdx.y * QG;
  const uint32_t nqg = (uint32_t)(nq - q0 < QG ? nq - q0 : QG);
  for (uint32_t i = threadIdx.x; i < QG * qpv; i += blockDim.x)
    sq[i] = i / qpv < nqg ? qbits[q0 * qpv + i] : 0ull;
  __syncthreads();
  for (uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; row < n;
       row += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t* d = words + row * qpv;
    uint32_t acc[QG];
#pragma unroll
    for (int g = 0; g < QG; g++) acc[g] = 0;
    for (uint32_t w0 = 0; w0 < qpv; w0 += 8) {
      uint64_t x[8];
      load_words8<VEC>(d + w0, qpv - w0, x);
#pragma unroll
      for (int i = 0; i < 8; i++) {
        if (w0 + i < qpv) {
#pragma unroll
          for (int g = 0; g < QG; g++) {
            const uint64_t qw = sq[g * qpv + w0 + i];
            acc[g] += __popcll(mode == 0 ? (x[i] ^ qw) : (x[i] & qw));
          }
        }
      }
    }
#pragma unroll
    for (int g = 0; g < QG; g++)
      if (g < (int)nqg) keys[(q0 + g) * ld + row] = mode == 0 ? acc[g] : n_top - acc[g];
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

// One lane per document: for each (a, b) with W[a,b] != 0 the exact integer
// overlap popcount(Q_a AND D_b) over the bucket's words, accumulated in f32 in
// (a, b) order exactly as the reference (acc += W[a,b] * overlap).  D_b's
// words are re-read from L1 for each a; query words and weights in shared
// memory.
template <bool VEC>
__global__ void __launch_bounds__(kThreads)
    multibucket_rows_kernel(const uint64_t* __restrict__ words, uint64_t n, uint32_t qpb,
                            uint32_t nb, const uint64_t* __restrict__ qbits,
                            const float* __restrict__ wts, uint32_t* __restrict__ keys,
                            uint64_t ld) {
  extern __shared__ uint64_t sm_mb[];  // nb * qpb query words, then nb * nb weights
  const uint64_t qi = blockIdx.y;
  const uint32_t per_doc = nb * qpb;
  float* sw = reinterpret_cast<float*>(sm_mb + per_doc);
  for (uint32_t i = threadIdx.x; i < per_doc; i += blockDim.x) sm_mb[i] = qbits[qi * per_doc + i];
  for (uint32_t i = threadIdx.x; i < nb * nb; i += blockDim.x) sw[i] = wts[i];
  __syncthreads();
  for (uint64_t doc = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; doc < n;
       doc += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t* d = words + doc * per_doc;
    float acc = 0.0f;
    for (uint32_t a = 0; a < nb; a++)
      for (uint32_t b = 0; b < nb; b++) {
        const float wt = sw[a * nb + b];
        if (wt == 0.0f) continue;
        uint32_t ov = 0;
        for (uint32_t w0 = 0; w0 < qpb; w0 += 8) {
          uint64_t x[8];
          load_words8<VEC>(d + b * qpb + w0, qpb - w0, x);
#pragma unroll
          for (int i = 0; i < 8; i++)
            if (w0 + i < qpb) ov += __popcll(sm_mb[a * qpb + w0 + i] & x[i]);
        }
        acc = __fadd_rn(acc, __fmul_rn(wt, (float)ov));
      }
    keys[qi * ld + doc] = desc_key(acc);
  }
}

unsigned scan_grid(uint64_t units_per_cta, uint64_t n) {
  uint64_t g = (n + units_per_cta - 1) / units_per_cta;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (unsigned)g;
}

template <int QG>
void launch_rows(int mode, const uint64_t* words, uint64_t n, uint32_t qpv, const uint64_t* qbits, uint64_t nq,
                 uint32_t n_top, uint32_t* keys, uint64_t ld, cudaStream_t stream) {
  const size_t smem = (size_t)QG * qpv * 8;
  // 16-byte loads when every row starts 16-byte aligned
  const bool vec = qpv % 2 == 0 && reinterpret_cast<uintptr_t>(words) % 16 == 0;
  auto kernel = vec ? popc_rows_kernel<QG, true> : popc_rows_kernel<QG, false>;
  allow_dynamic_smem(kernel);
  const uint64_t groups = (nq + QG - 1) / QG;
  for (uint64_t g0 = 0; g0 < groups; g0 += 65535) {
    const uint64_t gy = groups - g0 < 65535 ? groups - g0 : 65535;
    const dim3 grid(scan_grid(kThreads, n), (unsigned)gy);
    kernel<<<grid, kThreads, smem, stream>>>(mode, words, n, qpv, qbits + g0 * QG * qpv, nq - g0 * QG, n_top,
                                             keys + g0 * QG * ld, ld);
    launched();
  }
}

}  // namespace

void launch_popc_scan(int mode, const uint64_t* words, uint64_t n, uint32_t qpv,
                      const uint64_t* qbits, uint64_t nq, uint32_t n_top, uint32_t* keys,
                      uint64_t ld, cudaStream_t stream) {
  if (!n || !nq) return;
  if (8ull * qpv * 8 > 200 * 1024) throw std::invalid_argument("popcount scan: rows too long for the query stage");
  if (nq == 1)
    launch_rows<1>(mode, words, n, qpv, qbits, nq, n_top, keys, ld, stream);
  else if (nq == 2)
    launch_rows<2>(mode, words, n, qpv, qbits, nq, n_top, keys, ld, stream);
  else if (nq <= 4)
    launch_rows<4>(mode, words, n, qpv, qbits, nq, n_top, keys, ld, stream);
  else
    launch_rows<8>(mode, words, n, qpv, qbits, nq, n_top, keys, ld, stream);
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
  const size_t smem = (size_t)nb * qpb * 8 + (size_t)nb * nb * 4;
  const bool vec = qpb % 2 == 0 && reinterpret_cast<uintptr_t>(words) % 16 == 0;
  auto kernel = vec ? multibucket_rows_kernel<true> : multibucket_rows_kernel<false>;
  if (smem > 200 * 1024) throw std::invalid_argument("multi-bucket scan: rows too long");
  allow_dynamic_smem(kernel);
  for (uint64_t q0 = 0; q0 < nq; q0 += 65535) {
    unsigned gy = (unsigned)((nq - q0) < 65535 ? (nq - q0) : 65535);
    dim3 grid(scan_grid(kThreads, n), gy);
    kernel<<<grid, kThreads, smem, stream>>>(words, n, qpb, nb, qbits + q0 * (uint64_t)nb * qpb, w, keys + q0 * ld,
                                             ld);
    launched();
  }
}

}  // namespace ovb
