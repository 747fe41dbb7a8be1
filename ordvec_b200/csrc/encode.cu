// Device encoders for the `add` paths.
//
// rank_transform (src/rank.rs:38-53): ascending value, equal values (==, so
// -0.0 == +0.0) by ascending index.  Each document is one CTA: keys
// (asc_key(canonical value) << 32 | index) are bitonic-sorted in shared
// memory, sorted position = rank.  Emission per index family:
//   0 RankQuant   rank -> bucket floor(rank*2^b/dim) -> MSB-first pack
//                 (src/rank.rs:89-156, src/quant.rs:587-614)
//   1 SignBitmap  bit j = v[j] > 0 (src/sign_bitmap.rs:180-200), no sort
//   2 Bitmap      bit j = rank[j] >= dim - n_top (src/bitmap.rs:140-162)
//   3 FastScan    b=2 buckets, nibble (b[2p]<<2)|b[2p+1] (src/fastscan.rs:87-110),
//                 written straight into the device block layout (scan_fastscan.cu)
//   4 MultiBucket one bitmap per bucket (src/multi_bucket.rs:95-117)
//   5 Rank        the u16 rank itself (src/rank.rs:340-354)
//   6 symmetric RankQuant query: bucket_centre(bucket) as f32, the query side
//                 of RankQuant::search's LUT (src/quant.rs:660-669)
#include "ovb_common.cuh"
#include "ovb_kernels.h"

namespace ovb {

namespace {

__device__ void enc_bitonic(uint64_t* buf, uint32_t len) {
  for (uint32_t size = 2; size <= len; size <<= 1)
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t t = threadIdx.x; t < len / 2; t += blockDim.x) {
        uint32_t i = 2 * t - (t & (stride - 1)), j = i + stride;
        bool up = (i & size) == 0;
        uint64_t a = buf[i], b = buf[j];
        if ((a > b) == up) {
          buf[i] = b;
          buf[j] = a;
        }
      }
      __syncthreads();
    }
}

__global__ void rank_encode_kernel(int kind, const float* __restrict__ vecs, uint32_t dim,
                                   uint32_t bits, uint32_t n_top, uint32_t pairs_pad, uint32_t len,
                                   void* __restrict__ out, uint64_t first_doc) {
  extern __shared__ __align__(16) uint64_t sk[];
  uint16_t* rank = (uint16_t*)(sk + len);
  const uint64_t d = blockIdx.x;
  const float* v = vecs + d * dim;
  for (uint32_t j = threadIdx.x; j < len; j += blockDim.x) {
    if (j < dim) {
      float x = v[j];
      x = x == 0.0f ? 0.0f : x;
      sk[j] = ((uint64_t)asc_key(x) << 32) | j;
    } else {
      sk[j] = ~0ull;
    }
  }
  __syncthreads();
  enc_bitonic(sk, len);
  for (uint32_t p = threadIdx.x; p < dim; p += blockDim.x) rank[(uint32_t)sk[p]] = (uint16_t)p;
  __syncthreads();
  const uint64_t doc = first_doc + d;
  if (kind == 0) {
    const uint32_t cpb = 8 / bits, bpv = dim * bits / 8;
    uint8_t* o = (uint8_t*)out + doc * bpv;
    for (uint32_t t = threadIdx.x; t < bpv; t += blockDim.x) {
      uint32_t byte = 0;
      for (uint32_t i = 0; i < cpb; i++) {
        uint32_t j = t * cpb + i;
        uint32_t b = (uint32_t)(((uint64_t)rank[j] << bits) / dim);
        byte |= b << ((cpb - 1 - i) * bits);
      }
      o[t] = (uint8_t)byte;
    }
  } else if (kind == 2) {
    const uint32_t qpv = dim / 64, cutoff = dim - n_top;
    uint64_t* o = (uint64_t*)out + doc * qpv;
    for (uint32_t w = threadIdx.x; w < qpv; w += blockDim.x) {
      uint64_t word = 0;
      for (int j = 0; j < 64; j++)
        if (rank[w * 64 + j] >= cutoff) word |= 1ull << j;
      o[w] = word;
    }
  } else if (kind == 3) {
    const uint32_t pairs = dim / 2;
    const uint64_t blk = doc / 32, lane = doc % 32;
    uint8_t* o = (uint8_t*)out + blk * (uint64_t)pairs_pad * 16;
    for (uint32_t t = threadIdx.x; t < pairs_pad / 2; t += blockDim.x) {
      uint32_t g = t / 16, b = t % 16, nib[2];
      for (int h = 0; h < 2; h++) {
        uint32_t p = g * 32 + 2 * b + h;
        if (p < pairs) {
          uint32_t a = (uint32_t)(((uint64_t)rank[2 * p] << 2) / dim) & 3;
          uint32_t c = (uint32_t)(((uint64_t)rank[2 * p + 1] << 2) / dim) & 3;
          nib[h] = (a << 2) | c;
        } else {
          nib[h] = 0;
        }
      }
      o[(g * 32 + lane) * 16 + b] = (uint8_t)(nib[0] | (nib[1] << 4));
    }
  } else if (kind == 5) {
    uint16_t* o = (uint16_t*)out + doc * dim;
    for (uint32_t j = threadIdx.x; j < dim; j += blockDim.x) o[j] = rank[j];
  } else if (kind == 6) {
    float* o = (float*)out + doc * dim;
    const float centre = ((float)(1u << bits) - 1.0f) / 2.0f;
    for (uint32_t j = threadIdx.x; j < dim; j += blockDim.x)
      o[j] = (float)(uint32_t)(((uint64_t)rank[j] << bits) / dim) - centre;
  } else {  // kind 4
    const uint32_t qpb = dim / 64, nb = 1u << bits;
    uint64_t* o = (uint64_t*)out + doc * (uint64_t)nb * qpb;
    for (uint32_t t = threadIdx.x; t < nb * qpb; t += blockDim.x) {
      const uint32_t bucket = t / qpb, w = t % qpb;
      uint64_t word = 0;
      for (int j = 0; j < 64; j++) {
        uint32_t b = (uint32_t)(((uint64_t)rank[w * 64 + j] << bits) / dim);
        if (b == bucket) word |= 1ull << j;
      }
      o[t] = word;
    }
  }
}

__global__ void sign_encode_kernel(const float* __restrict__ vecs, uint64_t n, uint32_t dim,
                                   uint64_t* __restrict__ out, uint64_t first_doc) {
  const uint32_t qpv = dim / 64;
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * qpv) return;
  const uint64_t d = t / qpv, w = t % qpv;
  const float* x = vecs + d * dim + w * 64;
  uint64_t bits = 0;
  for (int j = 0; j < 64; j++)
    if (x[j] > 0.0f) bits |= 1ull << j;
  out[(first_doc + d) * qpv + w] = bits;
}

}  // namespace

void launch_multibucket_query(const float* q, uint64_t nq, uint32_t dim, uint32_t bits,
                              uint64_t* out, cudaStream_t stream) {
  launch_encode(4, q, nq, dim, bits, 0, 0, out, 0, stream);
}

void launch_encode(int kind, const float* vecs, uint64_t n, uint32_t dim, uint32_t bits,
                   uint32_t n_top, uint32_t pairs_pad, void* out, uint64_t first_doc,
                   cudaStream_t stream) {
  if (!n) return;
  if (kind == 1) {
    uint64_t total = n * (dim / 64);
    sign_encode_kernel<<<ceil_div(total, 256), 256, 0, stream>>>(vecs, n, dim, (uint64_t*)out, first_doc);
    launched();
    return;
  }
  uint32_t len = 1;
  while (len < dim) len <<= 1;
  const size_t smem = (size_t)len * 8 + (size_t)dim * 2;
  if (smem > 227 * 1024) throw std::invalid_argument("dim too large for the device rank transform");
  allow_dynamic_smem(rank_encode_kernel);
  const unsigned threads = len >= 1024 ? 512 : 256;
  for (uint64_t d0 = 0; d0 < n; d0 += 0x7FFFFFFF) {
    uint64_t cnt = n - d0 < 0x7FFFFFFF ? n - d0 : 0x7FFFFFFF;
    rank_encode_kernel<<<(unsigned)cnt, threads, smem, stream>>>(kind, vecs + d0 * dim, dim, bits, n_top,
                                                                 pairs_pad, len, out, first_doc + d0);
    launched();
  }
}

}  // namespace ovb
