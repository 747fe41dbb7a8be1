// K3 on the 5th-generation tensor cores: FastScan b=2 scoring of many queries
// at once as an exact integer GEMM.
//
//   acc[doc][q] = sum_p LUT_q[p][nib_p(doc)] = sum_k onehot(doc)[k] * LUT_q[k],
//   k = 16 p + nibble  (K = pairs_pad * 16 = 8192 at dim 1024)
//
// A (M = 128 docs x K) is the one-hot expansion of the nibble codes, built in
// shared memory by the CTA's threads; B (N = up to 256 queries x K) is the u8
// LUT matrix, loaded by TMA; D (128 x N, s32) accumulates in tensor memory with
// tcgen05.mma kind::i8 (u8 x u8).  Both operands use the K-major 128-byte
// swizzled layout: row r of a 128-byte K-block at (r/8)*1024 + (r%8)*128, its
// 16-byte chunk c at ((c ^ r%8) * 16).  The sum is exact, so the scores
//   (bias + (acc as f32) * inv_q) * inv_norm
// equal the CUDA-core kernel's (and the reference's) bit for bit.
//
// Pipeline: STAGES smem stages of (A 16 KiB + B up to 32 KiB); per K-block all
// threads expand A while thread 0 issues the B TMA, then thread 0 issues four
// K=32 MMAs and commits them to the stage's mbarrier, which the threads wait
// on before reusing the stage.  Every wait is bounded: on timeout the kernel
// records an error bit, stops issuing work, waits (bounded) for what it issued,
// frees its tensor memory and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "ovb_common.cuh"
#include "ovb_kernels.h"

namespace ovb {

namespace {

constexpr int kTcThreads = 128;
constexpr int kTcM = 128;
constexpr int kTcMaxN = 256;
constexpr int kTcKBytes = 128;  // 8 pairs x 16 one-hot bytes per K-block
constexpr int kTcStages = 3;
constexpr uint32_t kAStage = kTcM * kTcKBytes;       // 16 KiB
constexpr uint32_t kBStage = kTcMaxN * kTcKBytes;    // 32 KiB
constexpr uint32_t kTmemCols = 256;
constexpr uint32_t kWaitLimit = 1u << 22;

struct TcSmem {
  uint8_t a[kTcStages][kAStage];
  uint8_t b[kTcStages][kBStage];
  float bias[kTcMaxN];
  float invq[kTcMaxN];
  uint64_t mbar_tma[kTcStages];
  uint64_t mbar_mma[kTcStages];
  uint32_t tmem;
  uint32_t abort;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Bounded parity wait; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  for (uint32_t it = 0; it < kWaitLimit; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// K-major, 128-byte swizzle, 1024-byte atoms (8 rows x 128 B): LBO unused (1),
// SBO = 1024 B, version 1, layout type 2.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFF) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
        "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
        "=r"(v[30]), "=r"(v[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(kTcThreads, 1)
    fastscan_tc_kernel(const uint8_t* __restrict__ blocks, uint64_t n, uint32_t pairs_pad,
                       const __grid_constant__ CUtensorMap lut_map, const float* __restrict__ bias,
                       const float* __restrict__ invq, float inv_norm, uint64_t nq, uint32_t nt,
                       uint32_t* __restrict__ keys, uint64_t ld, uint32_t* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int t = threadIdx.x, warp = t >> 5;
  const uint64_t doc0 = (uint64_t)blockIdx.x * kTcM;
  const uint64_t q0 = (uint64_t)blockIdx.y * nt;
  const uint32_t nqt = (uint32_t)((nq - q0) < nt ? (nq - q0) : nt);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 0) {
    for (int s = 0; s < kTcStages; s++) {
      mbar_init(&S.mbar_tma[s], 1);
      mbar_init(&S.mbar_mma[s], 1);
    }
    S.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (uint32_t i = t; i < nt; i += kTcThreads) {
    S.bias[i] = i < nqt ? bias[q0 + i] : 0.0f;
    S.invq[i] = i < nqt ? invq[q0 + i] : 0.0f;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S.tmem;

  // instruction descriptor: D s32, A/B u8, K-major, N = nt, M = 128
  const uint32_t idesc = (2u << 4) | ((nt >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
  const uint32_t b_bytes = nt * kTcKBytes;

  const uint32_t r = t;  // A row = doc within the tile
  const uint64_t doc = doc0 + r;
  const uint64_t n_blocks = (n + 31) / 32;
  const uint64_t blk = doc / 32;
  const uint32_t dl = (uint32_t)(doc % 32);
  const bool row_valid = blk < n_blocks;
  const uint8_t* row_codes = blocks + blk * (uint64_t)pairs_pad * 16 + (uint64_t)dl * 16;
  const uint32_t n_kb = pairs_pad / 8;
  uint4 chunk = make_uint4(0, 0, 0, 0);
  uint32_t issued = 0;          // K-blocks whose MMAs were committed (thread 0)
  int pending_tma = -1;         // stage of a TMA whose wait timed out (thread 0)
  uint32_t pending_parity = 0;

  for (uint32_t kb = 0; kb < n_kb; kb++) {
    const uint32_t s = kb % kTcStages, it = kb / kTcStages;
    if (kb >= kTcStages && !mbar_wait(&S.mbar_mma[s], (it - 1) & 1)) atomicOr(&S.abort, 1u);
    __syncthreads();
    if (S.abort) break;
    if (t == 0) {
      mbar_expect_tx(&S.mbar_tma[s], b_bytes);
      tma_load_2d(S.b[s], &lut_map, (int)(kb * kTcKBytes), (int)q0, &S.mbar_tma[s]);
    }
    if ((kb & 3) == 0)
      chunk = row_valid ? *reinterpret_cast<const uint4*>(row_codes + (uint64_t)(kb >> 2) * 512)
                        : make_uint4(0, 0, 0, 0);
    const uint32_t w = (kb & 3) == 0 ? chunk.x : (kb & 3) == 1 ? chunk.y : (kb & 3) == 2 ? chunk.z : chunk.w;
    uint8_t* arow = S.a[s] + (r >> 3) * 1024 + (r & 7) * 128;
#pragma unroll
    for (uint32_t c = 0; c < 8; c++) {
      const uint32_t nib = (w >> (4 * c)) & 15;
      const uint32_t one = 1u << (8 * (nib & 3)), sel = nib >> 2;
      uint4 v = make_uint4(sel == 0 ? one : 0, sel == 1 ? one : 0, sel == 2 ? one : 0, sel == 3 ? one : 0);
      *reinterpret_cast<uint4*>(arow + ((c ^ (r & 7)) << 4)) = v;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) {
      if (!mbar_wait(&S.mbar_tma[s], it & 1)) {
        atomicOr(&S.abort, 1u);
        pending_tma = (int)s;
        pending_parity = it & 1;
      } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a_base = smem_u32(S.a[s]), b_base = smem_u32(S.b[s]);
#pragma unroll
        for (uint32_t j = 0; j < 4; j++)
          mma_i8(tmem, sw128_desc(a_base + 32 * j), sw128_desc(b_base + 32 * j), idesc, (kb | j) != 0);
        mma_commit(&S.mbar_mma[s]);
        issued = kb + 1;
      }
    }
  }
  // drain: a TMA whose wait timed out must land before the CTA exits, and the
  // last committed MMA group (which covers all earlier ones) must finish
  if (t == 0 && pending_tma >= 0) mbar_wait(&S.mbar_tma[pending_tma], pending_parity);
  __shared__ uint32_t s_issued;
  if (t == 0) s_issued = issued;
  __syncthreads();
  const uint32_t last = s_issued;
  bool ok = last == n_kb;
  if (last > 0 && !mbar_wait(&S.mbar_mma[(last - 1) % kTcStages], ((last - 1) / kTcStages) & 1)) ok = false;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!ok || S.abort) {
    if (t == 0) atomicOr(err, 1u);
  } else {
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    for (uint32_t cb = 0; cb < nt; cb += 32) {
      uint32_t v[32];
      tmem_ld32(tmem + lane_base + cb, v);
      if (doc < n) {
#pragma unroll
        for (uint32_t j = 0; j < 32; j++) {
          const uint32_t q = cb + j;
          if (q < nqt) {
            const float sc = __fmul_rn(__fadd_rn(S.bias[q], __fmul_rn(__uint2float_rn(v[j]), S.invq[q])), inv_norm);
            keys[(q0 + q) * ld + doc] = desc_key(sc);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
      throw CudaError("cuTensorMapEncodeTiled entry point unavailable");
    return (PFN_cuTensorMapEncodeTiled_v12000)p;
  }();
  return fn;
}

}  // namespace

size_t fastscan_tc_smem_bytes() { return sizeof(TcSmem) + 1024; }

void launch_fastscan_scan_tc(const uint8_t* blocks, uint64_t n, uint32_t pairs_pad, const uint8_t* lut,
                             const float* bias_sum, const float* inv_q, float inv_norm, uint64_t nq,
                             uint32_t* keys, uint64_t ld, uint32_t* err, cudaStream_t stream) {
  if (!n || !nq) return;
  const uint64_t k_bytes = (uint64_t)pairs_pad * 16;
  // N per tile: a multiple of 16 in [16, 256]
  uint32_t nt = nq >= kTcMaxN ? kTcMaxN : (uint32_t)((nq + 15) / 16 * 16);
  CUtensorMap map;
  cuuint64_t gdim[2] = {(cuuint64_t)k_bytes, (cuuint64_t)nq};
  cuuint64_t gstride[1] = {(cuuint64_t)k_bytes};
  cuuint32_t box[2] = {(cuuint32_t)kTcKBytes, (cuuint32_t)nt};
  cuuint32_t estride[2] = {1, 1};
  CUresult rc = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)lut, gdim, gstride, box, estride,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rc != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed for the FastScan LUT matrix");
  const size_t smem = fastscan_tc_smem_bytes();
  OVB_CUDA(cudaFuncSetAttribute(fastscan_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const uint64_t doc_tiles = (n + kTcM - 1) / kTcM;
  const uint64_t q_tiles = (nq + nt - 1) / nt;
  if (q_tiles > 65535 || doc_tiles > 0x7FFFFFFF)
    throw std::invalid_argument("FastScan tensor-core scan: grid too large; split the query batch");
  dim3 grid((unsigned)doc_tiles, (unsigned)q_tiles);
  fastscan_tc_kernel<<<grid, kTcThreads, smem, stream>>>(blocks, n, pairs_pad, map, bias_sum, inv_q, inv_norm, nq,
                                                         nt, keys, ld, err);
  launched();
}

}  // namespace ovb
