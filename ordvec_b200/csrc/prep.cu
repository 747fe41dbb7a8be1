// K8: per-query preparation on the device, bit-exact with the reference.
//
// * l2_normalise  (src/util.rs:93-115): sequential f32 sum of squares from
//   -0.0, correctly rounded sqrt and reciprocal, elementwise multiply.  The
//   sum is sequential on purpose: the FastScan LUT (and with it every
//   candidate id) depends on q_unit bit for bit.
// * sign query    (src/sign_bitmap.rs:204-214): bit j set iff q[j] > 0.
// * bitmap query  (src/bitmap.rs:170-187): the n_top largest coordinates,
//   stable descending sort (ties keep the lower index; -0.0 == +0.0).
// * FastScan LUT  (src/fastscan.rs:130-173): v = qa*c[a] + qc*c[c] without
//   contraction, global min/max with first-occurrence ties, affine u8
//   quantisation with round-half-away-from-zero and clamp.
// The arithmetic uses explicit __f*_rn intrinsics so no FMA contraction or
// fast-math rewrite can change a bit.
#include "ovb_common.cuh"
#include "ovb_kernels.h"

namespace ovb {

namespace {

// One warp per query.  The warp squares the query into shared memory in
// 1024-element chunks; lane 0 then adds the squares in index order (the
// reference's sequential f32 sum) with loads four at a time, so the chain is
// bound by the add latency, not by memory latency.
__global__ void l2_normalise_kernel(const float* __restrict__ q, uint64_t nq, uint32_t dim,
                                    float* __restrict__ out) {
  __shared__ __align__(16) float sq[8][1024];
  const int wid = threadIdx.x / 32;
  const uint64_t qi = (uint64_t)blockIdx.x * (blockDim.x / 32) + wid;
  const int lane = threadIdx.x & 31;
  if (qi >= nq) return;
  const float* x = q + qi * dim;
  float* y = out + qi * dim;
  float s = -0.0f;
  for (uint32_t c0 = 0; c0 < dim; c0 += 1024) {
    const uint32_t cn = dim - c0 < 1024 ? dim - c0 : 1024;
    for (uint32_t j = lane; j < cn; j += 32) sq[wid][j] = __fmul_rn(x[c0 + j], x[c0 + j]);
    __syncwarp();
    if (lane == 0) {
      uint32_t j = 0;
      for (; j + 4 <= cn; j += 4) {
        const float4 v = *reinterpret_cast<const float4*>(&sq[wid][j]);
        s = __fadd_rn(s, v.x);
        s = __fadd_rn(s, v.y);
        s = __fadd_rn(s, v.z);
        s = __fadd_rn(s, v.w);
      }
      for (; j < cn; j++) s = __fadd_rn(s, sq[wid][j]);
    }
    __syncwarp();
  }
  s = __shfl_sync(0xFFFFFFFFu, s, 0);
  const float norm = __fsqrt_rn(s);
  if (norm <= 1e-12f) {
    for (uint32_t j = lane; j < dim; j += 32) y[j] = 0.0f;
  } else {
    const float inv = __fdiv_rn(1.0f, norm);
    for (uint32_t j = lane; j < dim; j += 32) y[j] = __fmul_rn(x[j], inv);
  }
}

__global__ void sign_query_kernel(const float* __restrict__ q, uint64_t nq, uint32_t dim,
                                  uint64_t* __restrict__ out) {
  const uint32_t qpv = dim / 64;
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq * qpv) return;
  const uint64_t qi = t / qpv, w = t % qpv;
  const float* x = q + qi * dim + w * 64;
  uint64_t bits = 0;
  for (int j = 0; j < 64; j++)
    if (x[j] > 0.0f) bits |= 1ull << j;
  out[t] = bits;
}

// Bitonic sort of `len` (power of two) u64 keys in shared memory.
__device__ void block_bitonic(uint64_t* buf, uint32_t len) {
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

__device__ __forceinline__ float canon_zero(float v) { return v == 0.0f ? 0.0f : v; }

// n_top largest coordinates, stable: key = (desc value, index) ascending.
__global__ void bitmap_query_kernel(const float* __restrict__ q, uint32_t dim, uint32_t n_top,
                                    uint32_t len, uint64_t* __restrict__ out) {
  extern __shared__ uint64_t skeys[];
  const float* x = q + (uint64_t)blockIdx.x * dim;
  for (uint32_t j = threadIdx.x; j < len; j += blockDim.x)
    skeys[j] = j < dim ? ((uint64_t)desc_key(canon_zero(x[j])) << 32) | j : ~0ull;
  __syncthreads();
  block_bitonic(skeys, len);
  const uint32_t qpv = dim / 64;
  uint64_t* o = out + (uint64_t)blockIdx.x * qpv;
  for (uint32_t w = threadIdx.x; w < qpv; w += blockDim.x) o[w] = 0;
  __syncthreads();
  for (uint32_t t = threadIdx.x; t < n_top; t += blockDim.x) {
    uint32_t j = (uint32_t)skeys[t];
    atomicOr((unsigned long long*)&o[j / 64], 1ull << (j % 64));
  }
}

struct MinMax {
  float mn, mx;
  uint32_t imn, imx;
};

__device__ __forceinline__ float fs_value(const float* qu, uint32_t i) {
  const uint32_t p = i >> 4, a = (i >> 2) & 3, c = i & 3;
  // bucket_centre(b, 2) = b - 1.5: exactly -1.5, -0.5, 0.5, 1.5
  const float ca = (float)a - 1.5f, cc = (float)c - 1.5f;
  return __fadd_rn(__fmul_rn(qu[2 * p], ca), __fmul_rn(qu[2 * p + 1], cc));
}

__global__ void fastscan_lut_kernel(const float* __restrict__ q_unit, uint32_t dim,
                                    uint32_t pairs_pad, uint8_t* __restrict__ lut,
                                    float* __restrict__ bias_sum, float* __restrict__ inv_q) {
  __shared__ MinMax part[32];
  __shared__ float s_gmin, s_scale;
  const uint32_t pairs = dim / 2, total = pairs * 16;
  const float* qu = q_unit + (uint64_t)blockIdx.x * dim;
  // sequential semantics per thread (ascending index, strict compares)
  MinMax m{__int_as_float(0x7f800000), __int_as_float(0xff800000), 0xFFFFFFFFu, 0xFFFFFFFFu};
  for (uint32_t i = threadIdx.x; i < total; i += blockDim.x) {
    float v = fs_value(qu, i);
    if (v < m.mn) { m.mn = v; m.imn = i; }
    if (v > m.mx) { m.mx = v; m.imx = i; }
  }
  // combine: value order, first index on equality (== treats -0 and +0 alike)
  for (int o = 16; o > 0; o >>= 1) {
    MinMax r;
    r.mn = __shfl_down_sync(0xFFFFFFFFu, m.mn, o);
    r.imn = __shfl_down_sync(0xFFFFFFFFu, m.imn, o);
    r.mx = __shfl_down_sync(0xFFFFFFFFu, m.mx, o);
    r.imx = __shfl_down_sync(0xFFFFFFFFu, m.imx, o);
    if (r.imn != 0xFFFFFFFFu && (m.imn == 0xFFFFFFFFu || r.mn < m.mn || (r.mn == m.mn && r.imn < m.imn))) {
      m.mn = r.mn;
      m.imn = r.imn;
    }
    if (r.imx != 0xFFFFFFFFu && (m.imx == 0xFFFFFFFFu || r.mx > m.mx || (r.mx == m.mx && r.imx < m.imx))) {
      m.mx = r.mx;
      m.imx = r.imx;
    }
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) part[w] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    MinMax g = part[0];
    for (int i = 1; i < (int)(blockDim.x / 32); i++) {
      MinMax r = part[i];
      if (r.imn != 0xFFFFFFFFu && (g.imn == 0xFFFFFFFFu || r.mn < g.mn || (r.mn == g.mn && r.imn < g.imn))) {
        g.mn = r.mn;
        g.imn = r.imn;
      }
      if (r.imx != 0xFFFFFFFFu && (g.imx == 0xFFFFFFFFu || r.mx > g.mx || (r.mx == g.mx && r.imx < g.imx))) {
        g.mx = r.mx;
        g.imx = r.imx;
      }
    }
    float span = __fsub_rn(g.mx, g.mn);
    if (!(span >= 1e-12f)) span = 1e-12f;
    const float scale = __fdiv_rn(255.0f, span);
    s_gmin = g.mn;
    s_scale = scale;
    inv_q[blockIdx.x] = __fdiv_rn(1.0f, scale);
    bias_sum[blockIdx.x] = __fmul_rn((float)pairs, g.mn);
  }
  __syncthreads();
  const float gmin = s_gmin, scale = s_scale;
  uint8_t* L = lut + (uint64_t)blockIdx.x * pairs_pad * 16;
  for (uint32_t i = threadIdx.x; i < pairs_pad * 16; i += blockDim.x) {
    uint8_t u = 0;
    if (i < total) {
      float r = roundf(__fmul_rn(__fsub_rn(fs_value(qu, i), gmin), scale));
      r = r < 0.0f ? 0.0f : (r > 255.0f ? 255.0f : r);
      u = (uint8_t)r;
    }
    L[i] = u;
  }
}

// assert_all_finite (src/util.rs:126-141) on the device: sets *flag if any
// value is NaN or +-Inf.
__global__ void finite_flag_kernel(const float* __restrict__ x, uint64_t count,
                                   uint32_t* __restrict__ flag) {
  bool bad = false;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x)
    bad |= !isfinite(x[i]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1u);
}

__global__ void uniform_offsets_kernel(uint64_t* off, uint64_t nq, uint64_t m) {
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t <= nq) off[t] = t * m;
}

__global__ void keys_to_results_kernel(const uint32_t* __restrict__ keys,
                                       const uint32_t* __restrict__ ids, uint64_t count,
                                       int mode, uint32_t n_top, float* __restrict__ scores,
                                       int64_t* __restrict__ out_ids) {
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  uint32_t k = keys[t], id = ids[t];
  if (id == kSentinelId) {
    scores[t] = __int_as_float(0xff800000);
    out_ids[t] = -1;
    return;
  }
  scores[t] = mode == 0 ? desc_key_to_float(k) : (float)(n_top - k);
  out_ids[t] = (int64_t)id;
}

}  // namespace

void launch_l2_normalise(const float* q, uint64_t nq, uint32_t dim, float* out,
                         cudaStream_t stream) {
  if (!nq) return;
  l2_normalise_kernel<<<ceil_div(nq, 8), 256, 0, stream>>>(q, nq, dim, out);
  launched();
}

void launch_sign_query(const float* q, uint64_t nq, uint32_t dim, uint64_t* out,
                       cudaStream_t stream) {
  uint64_t total = nq * (dim / 64);
  if (!total) return;
  sign_query_kernel<<<ceil_div(total, 256), 256, 0, stream>>>(q, nq, dim, out);
  launched();
}

void launch_bitmap_query(const float* q, uint64_t nq, uint32_t dim, uint32_t n_top,
                         uint64_t* out, cudaStream_t stream) {
  if (!nq) return;
  uint32_t len = 1;
  while (len < dim) len <<= 1;
  size_t smem = (size_t)len * 8;
  if (smem > 227 * 1024) throw std::invalid_argument("Bitmap query dim too large for the device path (dim <= 16384)");
  allow_dynamic_smem(bitmap_query_kernel);
  bitmap_query_kernel<<<(unsigned)nq, 512, smem, stream>>>(q, dim, n_top, len, out);
  launched();
}

void launch_fastscan_lut(const float* q_unit, uint64_t nq, uint32_t dim, uint32_t pairs_pad,
                         uint8_t* lut, float* bias_sum, float* inv_q, cudaStream_t stream) {
  if (!nq) return;
  // one CTA per query; a lone query (one-query calls) gets the widest CTA
  fastscan_lut_kernel<<<(unsigned)nq, nq <= 16 ? 1024 : 256, 0, stream>>>(q_unit, dim, pairs_pad, lut, bias_sum,
                                                                          inv_q);
  launched();
}

void launch_finite_flag(const float* x, uint64_t count, uint32_t* flag, cudaStream_t stream) {
  if (!count) return;
  uint64_t blocks = (count + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  finite_flag_kernel<<<(unsigned)blocks, 256, 0, stream>>>(x, count, flag);
  launched();
}

namespace {
// Row q's first off[q+1] - off[q] entries of src (row stride ld) -> dst[off[q] ..]
__global__ void prefix_compact_kernel(const uint32_t* __restrict__ src, uint64_t ld, const uint64_t* __restrict__ off,
                                      uint32_t* __restrict__ dst) {
  const uint64_t q = blockIdx.x;
  const uint64_t a = off[q], len = off[q + 1] - a;
  for (uint64_t j = threadIdx.x; j < len; j += blockDim.x) dst[a + j] = src[q * ld + j];
}

__global__ void clamp_ids_kernel(uint32_t* ids, uint64_t count, uint32_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
    if (ids[i] >= n) ids[i] = 0;
}
}  // namespace

void launch_clamp_ids(uint32_t* ids, uint64_t count, uint32_t n, cudaStream_t stream) {
  if (!count) return;
  uint64_t blocks = ceil_div(count, 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  clamp_ids_kernel<<<(unsigned)blocks, 256, 0, stream>>>(ids, count, n);
  launched();
}

void launch_prefix_compact(const uint32_t* src, uint64_t ld, const uint64_t* off, uint64_t nq, uint32_t* dst,
                           cudaStream_t stream) {
  if (!nq) return;
  if (nq > 0x7FFFFFFFull) throw std::invalid_argument("prefix compaction: too many rows");
  prefix_compact_kernel<<<(unsigned)nq, 256, 0, stream>>>(src, ld, off, dst);
  launched();
}

void launch_uniform_offsets(uint64_t* off, uint64_t nq, uint64_t m, cudaStream_t stream) {
  uniform_offsets_kernel<<<ceil_div(nq + 1, 256), 256, 0, stream>>>(off, nq, m);
  launched();
}

void launch_keys_to_results(const uint32_t* keys, const uint32_t* ids, uint64_t count,
                            int mode, uint32_t n_top, float* scores, int64_t* out_ids,
                            cudaStream_t stream) {
  if (!count) return;
  keys_to_results_kernel<<<ceil_div(count, 256), 256, 0, stream>>>(keys, ids, count, mode, n_top, scores, out_ids);
  launched();
}

}  // namespace ovb
