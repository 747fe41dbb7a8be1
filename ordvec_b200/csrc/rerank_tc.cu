// K5-TC: the split-BF16 candidate rerank on the 5th-generation tensor cores.
//
// The reference reranks each query's candidate rows with its asymmetric
// scorer (RankQuant::search_asymmetric_subset, src/quant.rs:1048-1083 and
// subset_rerank_row_into :1126-1281):
//
//   s(q, d) = inv_norm * sum_j q_j * (code_j - c),   c = (2^B - 1) / 2.
//
// Here every (query, 128-candidate tile) is one CTA and the sum is a dense
// contraction on tcgen05 (kind::f16, f32 accumulation in TMEM):
//   A (M = 128 rows): the tile's candidate code rows, gathered from HBM into
//     shared memory by the builder threads (16-byte cp.async copies spread
//     over all 256 of them), then expanded by those 8 warps (two threads per row) into
//     the exact centred codes as bf16 (split_bf16.cuh), 64 coordinates per
//     128-byte-swizzled K-block, 3 K-block stages;
//   B (N = 16 rows, TMA): rows 2q .. 2q+15 of the [2 nq x dim] split query
//     matrix, of which rows 2q (hi = bf16(q)) and 2q+1 (lo = bf16(q - hi))
//     are the CTA's query; the other rows' columns are not read;
//   D: column 0 = hi . a, column 1 = lo . a; score = (acc_hi + acc_lo) *
//     inv_norm, rounded to nearest at each step.
// The result differs from the exact score by at most split_error_bound() *
// |q|_1 (the same bound as the split-BF16 scan); the engine keeps ids exact
// by rescoring every candidate within twice that bound of the k-th in FP64.
//
// Warp roles: warp 0 issues the B TMA loads, warp 1 issues the MMAs, warps
// 2..9 gather the rows, build A and then (warps 2..5, one TMEM lane
// quadrant each) run the epilogue.  Every wait is bounded: a timeout sets
// *err, drains the copies and MMAs in flight, frees TMEM and returns.
#include <cuda_bf16.h>

#include "ovb_common.cuh"
#include "ovb_kernels.h"
#include "split_bf16.cuh"
#include "tc_common.cuh"

namespace ovb {

namespace {

using namespace tc;

constexpr int kRrBuilders = 256;  // warps 2..9
constexpr int kRrThreads = 64 + kRrBuilders;
constexpr int kRrM = 128;       // candidate rows per CTA
constexpr int kRrN = 16;        // B rows per MMA
constexpr int kRrKBytes = 128;  // 64 bf16 coordinates per K-block
constexpr int kRrStages = 3;
constexpr uint32_t kRrAStage = kRrM * kRrKBytes;  // 16 KiB
constexpr uint32_t kRrBStage = kRrN * kRrKBytes;  // 2 KiB
constexpr uint32_t kRrRowStride = 272;            // staged row pitch (bytes): 16-byte aligned, 4-bank skew
constexpr uint32_t kRrTmemCols = 32;

struct RrSmem {
  uint8_t a[kRrStages][kRrAStage];
  uint8_t b[kRrStages][kRrBStage];
  uint8_t rows[kRrM][kRrRowStride];
  uint64_t full_a[kRrStages];
  uint64_t full_b[kRrStages];
  uint64_t empty[kRrStages];
  uint64_t acc_full;
  uint32_t tmem;
  uint32_t abort;
};

struct RrArgs {
  const uint8_t* codes;
  uint64_t n;
  uint32_t dim;
  uint32_t bpv;  // packed row bytes
  uint64_t nq;
  const uint32_t* cands;  // row q: cands[q * ld + j], j < m
  uint64_t ld;
  uint32_t m;
  uint32_t tiles;  // ceil(m / 128) CTAs per query
  float inv_norm;
  uint32_t* keys;  // keys[q * ld + j] = desc_key(split score)
  uint32_t* err;
};

__device__ __forceinline__ void rr_abort(RrSmem& S, uint32_t* err) {
  atomicExch(&S.abort, 1u);
  atomicOr(err, 1u);
}

__device__ __forceinline__ bool rr_aborted(const RrSmem& S) {
  return *reinterpret_cast<const volatile uint32_t*>(&S.abort) != 0;
}

// named barrier 2 over the builder warps
__device__ __forceinline__ void rr_build_sync() { asm volatile("bar.sync 2, %0;" ::"n"(kRrBuilders) : "memory"); }

__device__ __forceinline__ void tmem_ld2(uint32_t taddr, uint32_t& v0, uint32_t& v1) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(v0), "=r"(v1) : "r"(taddr) : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Lane-wait helper for the builders and the epilogue: lane 0 polls, the warp
// follows its verdict.
__device__ __forceinline__ bool warp_wait(uint64_t* bar, uint32_t parity, uint32_t lane) {
  bool ok = true;
  if (lane == 0) ok = mbar_wait(bar, parity);
  ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
  __syncwarp();
  return ok;
}

template <int BITS>
__global__ void __launch_bounds__(kRrThreads, 2)
    rerank_tc_kernel(const __grid_constant__ CUtensorMap q_map, const RrArgs a) {
  extern __shared__ uint8_t smem_raw[];
  RrSmem& S = *reinterpret_cast<RrSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const uint64_t q = blockIdx.x / a.tiles;
  const uint32_t j0 = (blockIdx.x % a.tiles) * kRrM;  // first candidate of the tile
  const uint32_t rows = a.m - j0 < (uint32_t)kRrM ? a.m - j0 : (uint32_t)kRrM;
  const uint32_t n_kb = a.dim / 64;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                 "r"(kRrTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 32) {
    for (int s = 0; s < kRrStages; s++) {
      mbar_init(&S.full_a[s], kRrBuilders / 32);
      mbar_init(&S.full_b[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    mbar_init(&S.acc_full, 1);
    S.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S.tmem;

  if (warp == 0) {
    // ---- B: this query's hi/lo rows (and 14 unread neighbours), one K-block per stage
    if (lane == 0) {
      uint32_t issued = 0;
      for (uint32_t kb = 0; kb < n_kb; kb++) {
        const uint32_t s = kb % kRrStages, it = kb / kRrStages;
        if (rr_aborted(S)) break;
        if (kb >= kRrStages && !mbar_wait(&S.empty[s], (it - 1) & 1)) {
          rr_abort(S, a.err);
          break;
        }
        mbar_expect_tx(&S.full_b[s], kRrBStage);
        tma_load_2d(S.b[s], &q_map, (int)(kb * 64), (int)(2 * q), &S.full_b[s]);
        issued = kb + 1;
      }
      // drain: no copy may land after the CTA has exited
      for (uint32_t kb = issued > kRrStages ? issued - kRrStages : 0; kb < issued; kb++)
        mbar_wait(&S.full_b[kb % kRrStages], (kb / kRrStages) & 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // D f32, A/B bf16, both K-major, N = 16, M = 128
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kRrN >> 3) << 17) |
                             ((uint32_t)(kRrM >> 4) << 24);
      uint32_t done = 0;
      for (uint32_t kb = 0; kb < n_kb; kb++) {
        const uint32_t s = kb % kRrStages, it = kb / kRrStages;
        if (rr_aborted(S)) break;
        if (!mbar_wait(&S.full_b[s], it & 1) || !mbar_wait(&S.full_a[s], it & 1)) {
          rr_abort(S, a.err);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_u32(S.a[s]), b0 = smem_u32(S.b[s]);
#pragma unroll
        for (uint32_t j = 0; j < 4; j++)
          mma_f16(tmem, sw128_desc(a0 + 32 * j), sw128_desc(b0 + 32 * j), idesc, (kb | j) != 0);
        mma_commit(&S.empty[s]);
        done = kb + 1;
      }
      if (done == n_kb && !rr_aborted(S)) {
        mma_commit(&S.acc_full);
        mbar_wait(&S.acc_full, 0);
      } else if (done > 0) {
        mbar_wait(&S.empty[(done - 1) % kRrStages], ((done - 1) / kRrStages) & 1);
      }
    }
  } else {
    // ---- A builders: row r, coordinates 32 hc .. 32 hc + 31 of each K-block
    const uint32_t bt = (uint32_t)t - 64;
    const uint32_t r = bt & (kRrM - 1), hc = bt >> 7;
    {
      // gather the tile's rows: 16-byte copies spread over the builders (ids clamped into range)
      const uint32_t cpr = a.bpv / 16;  // 16-byte chunks per row
      const uint32_t* ids = a.cands + q * a.ld + j0;
      for (uint32_t c = bt; c < rows * cpr; c += kRrBuilders) {
        const uint32_t rr = c / cpr, part = c - rr * cpr;
        uint32_t id = __ldg(ids + rr);
        if (id >= a.n) id = (uint32_t)(a.n - 1);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(S.rows[rr] + 16 * part)),
                     "l"(a.codes + (uint64_t)id * a.bpv + 16 * part)
                     : "memory");
      }
      asm volatile("cp.async.wait_all;" ::: "memory");
      rr_build_sync();
    }
    uint32_t t0, t1;
    nibble_table<BITS>((uint32_t)lane, t0, t1);
    const uint32_t a_row = smem_u32(S.a[0]) + (r >> 3) * 1024 + (r & 7) * 128;
    uint32_t dst[4];
#pragma unroll
    for (uint32_t c = 0; c < 4; c++) dst[c] = a_row + (((4 * hc + c) ^ (r & 7)) << 4);
    // rows past the tile's end are built from row 0 (their scores are not written)
    const uint8_t* src = S.rows[r < rows ? r : 0] + hc * 4 * BITS;
    bool ok = true;
    uint32_t s = 0, par = 0, base = 0;
    for (uint32_t kb = 0; kb < n_kb && ok && !rr_aborted(S); kb++) {
      if (kb >= (uint32_t)kRrStages) {
        ok = warp_wait(&S.empty[s], par ^ 1, (uint32_t)lane);
        if (!ok) {
          if (lane == 0) rr_abort(S, a.err);
          break;
        }
      }
      uint32_t w[4] = {0, 0, 0, 0};
      const uint8_t* p = src + kb * 8 * BITS;
      if (BITS == 4) {
        const uint4 v = *reinterpret_cast<const uint4*>(p);
        w[0] = v.x, w[1] = v.y, w[2] = v.z, w[3] = v.w;
      } else if (BITS == 2) {
        const uint2 v = *reinterpret_cast<const uint2*>(p);
        w[0] = v.x, w[1] = v.y;
      } else {
        w[0] = *reinterpret_cast<const uint32_t*>(p);
      }
#pragma unroll
      for (uint32_t c = 0; c < 4; c++) {  // 16-byte chunk c = coordinates 8c .. 8c+7
        uint32_t o[4];
        if (BITS == 2) {
#pragma unroll
          for (int i = 0; i < 4; i++) o[i] = __shfl_sync(0xFFFFFFFFu, t0, nib(w[c >> 1], 4 * (c & 1) + i));
        } else if (BITS == 1) {
#pragma unroll
          for (int i = 0; i < 2; i++) {
            const uint32_t v = nib(w[0], 2 * c + i);
            o[2 * i] = __shfl_sync(0xFFFFFFFFu, t0, v);
            o[2 * i + 1] = __shfl_sync(0xFFFFFFFFu, t1, v);
          }
        } else {
#pragma unroll
          for (int i = 0; i < 4; i++)
            o[i] = __shfl_sync(0xFFFFFFFFu, t0, nib(w[c], 2 * i)) | (__shfl_sync(0xFFFFFFFFu, t0, nib(w[c], 2 * i + 1)) << 16);
        }
        st_shared_v4(dst[c] + base, o[0], o[1], o[2], o[3]);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&S.full_a[s]);
      base += kRrAStage;
      if (++s == kRrStages) {
        s = 0;
        base = 0;
        par ^= 1;
      }
    }

    // ---- epilogue (warps 2..5: TMEM lane quadrant warp % 4)
    if (warp < 6) {
      bool ready = false;
      if (lane == 0) {
        const uint32_t addr = smem_u32(&S.acc_full);
        uint64_t c0 = 0;
        for (uint32_t it = 0; it < kWaitLimit && !rr_aborted(S); it++) {
          if (mbar_try(addr, 0)) {
            ready = true;
            break;
          }
          if ((it & 255) == 255) {
            const uint64_t now = global_ns();
            if (!c0)
              c0 = now;
            else if (now - c0 > kWaitNs)
              break;
          }
        }
        if (!ready && !rr_aborted(S)) rr_abort(S, a.err);
      }
      ready = __shfl_sync(0xFFFFFFFFu, ready, 0);
      __syncwarp();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (ready) {
        const uint32_t lq = (uint32_t)warp & 3, row = lq * 32 + lane;
        uint32_t hi, lo;
        tmem_ld2(tmem + ((lq * 32) << 16), hi, lo);
        if (row < rows)
          a.keys[q * a.ld + j0 + row] =
              desc_key(__fmul_rn(__fadd_rn(__uint_as_float(hi), __uint_as_float(lo)), a.inv_norm));
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kRrTmemCols) : "memory");
}

}  // namespace

bool rerank_tc_eligible(uint32_t dim, uint32_t bits) {
  const uint32_t bpv = dim * bits / 8;
  return rank_tc_eligible(dim, bits) && bpv % 16 == 0 && bpv <= kRrRowStride - 16;
}

void launch_rerank_tc(const uint8_t* codes, uint64_t n, uint32_t dim, uint32_t bits, const void* q_split,
                      uint64_t nq, const uint32_t* cands, uint64_t ld, uint32_t m, float inv_norm, uint32_t* keys,
                      uint32_t* err, cudaStream_t stream) {
  if (!n || !nq || !m) return;
  if (!rerank_tc_eligible(dim, bits))
    throw std::invalid_argument("split-BF16 rerank: needs dim % 64 == 0 and 16 <= bytes per row <= 256");
  if (m > ld) throw std::invalid_argument("split-BF16 rerank: row length exceeds the row stride");
  RrArgs a{};
  a.codes = codes;
  a.n = n;
  a.dim = dim;
  a.bpv = dim * bits / 8;
  a.nq = nq;
  a.cands = cands;
  a.ld = ld;
  a.m = m;
  a.tiles = (m + kRrM - 1) / kRrM;
  a.inv_norm = inv_norm;
  a.keys = keys;
  a.err = err;
  const uint64_t ctas = nq * a.tiles;
  if (ctas > 0x7FFFFFFFull) throw std::invalid_argument("split-BF16 rerank: grid too large; split the query batch");
  CUtensorMap map;
  cuuint64_t gdim[2] = {(cuuint64_t)dim, (cuuint64_t)(2 * nq)};
  cuuint64_t gstride[1] = {(cuuint64_t)dim * 2};
  cuuint32_t box[2] = {64, (cuuint32_t)kRrN};
  cuuint32_t estride[2] = {1, 1};
  CUresult rc = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(q_split), gdim, gstride, box,
                            estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rc != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed for the split query matrix");
  const size_t smem = sizeof(RrSmem) + 1024;
#define OVB_RR(B)                                                                                                \
  do {                                                                                                           \
    allow_dynamic_smem(rerank_tc_kernel<B>);                                                                    \
    rerank_tc_kernel<B><<<(unsigned)ctas, kRrThreads, smem, stream>>>(map, a);                                  \
  } while (0)
  if (bits == 1)
    OVB_RR(1);
  else if (bits == 2)
    OVB_RR(2);
  else
    OVB_RR(4);
#undef OVB_RR
  launched();
}

}  // namespace ovb
