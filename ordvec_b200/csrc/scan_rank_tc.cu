// K4-TC: asymmetric RankQuant scores of many queries on the 5th-generation
// tensor cores, split-BF16:
//
//   s(q, d) = inv_norm * sum_j q_j * (code_j - c),   c = (2^B - 1) / 2
//
// A (256 docs per CTA as two M=128 accumulators, K = dim): the centred codes
// (code - c) as bf16.  They are exact: (2 code - 2^B + 1) / 2 has at most 4
// significant bits.  Builder warps expand the packed rows (MSB-first codes)
// in shared memory through a 16-entry nibble table that lives in the lanes
// of each warp and is read with warp shuffles: one shuffle per 4-bit group
// of codes yields their bf16 pair (b=2), pair of pairs (b=1) or value (b=4).
// B: two rows per query, hi = bf16(q) and lo = bf16(q - hi) (so hi + lo
// carries 16 significant bits of q), loaded by TMA from a [2 nq x dim] bf16
// matrix.  D (f32, TMEM): column 2i = q_i.hi . a, column 2i+1 = q_i.lo . a;
// every product is exact in f32 and the tensor core accumulates in f32.
// score = (acc_hi + acc_lo) * inv_norm, rounded to nearest at each step.
//
// The result differs from the exact (FP64) score by at most the bound
// split_error_bound() states; callers that need exact top-k rescore the
// candidates within twice that bound of the k-th score in FP64.
//
// Pipeline and fault handling are the FastScan tensor-core kernel's: warp 0
// issues the B TMA loads, warp 1 the MMAs, warps 2..17 build A (two threads
// per doc row) and then run the epilogue; 3 stages of (A 32 KiB + B 32 KiB);
// every wait is bounded and a timeout sets *err, drains and frees TMEM.
#include <cuda_bf16.h>

#include "ovb_common.cuh"
#include "ovb_kernels.h"
#include "split_bf16.cuh"
#include "tc_common.cuh"

namespace ovb {

namespace {

using namespace tc;

constexpr int kRtThreads = 576;
constexpr int kRtBuilders = 512;  // warps 2..17
constexpr int kRtM = 256;         // docs per CTA
constexpr int kRtMaxN = 256;      // B rows per tile (128 queries)
constexpr int kRtKBytes = 128;    // 64 bf16 coordinates per K-block
constexpr int kRtStages = 3;
constexpr uint32_t kRtAHalf = 128 * kRtKBytes;
constexpr uint32_t kRtAStage = kRtM * kRtKBytes;
constexpr uint32_t kRtBStage = kRtMaxN * kRtKBytes;
constexpr uint32_t kRtTmemCols = 512;
constexpr uint32_t kRtAcc1Col = 256;

constexpr uint32_t kRtMaxQ = kRtMaxN / 2;  // queries per tile
// filter list (key, q | slot << 8 | row << 16) in the dead A stages, one segment per epilogue warp
constexpr uint32_t kRtSegCap = kRtStages * kRtAStage / 8 / (kRtBuilders / 32);

struct RtSmem {
  uint8_t a[kRtStages][kRtAStage];
  uint8_t b[kRtStages][kRtBStage];
  uint32_t thr[kRtMaxQ];
  uint32_t cnt[kRtMaxQ];
  uint32_t base[kRtMaxQ];
  uint64_t full_a[kRtStages];
  uint64_t full_b[kRtStages];
  uint64_t empty[kRtStages];
  uint64_t acc_full;
  uint32_t tmem;
  uint32_t abort;
  uint32_t epi_ok;
  uint32_t seg_full;
};

struct RtArgs {
  const uint8_t* codes;
  uint64_t n;
  uint32_t dim;
  uint32_t bpv;  // bytes per packed row
  uint64_t nq;
  uint32_t nt;  // B rows per tile (2 per query)
  uint32_t q_tiles;  // query tiles; CTA b covers query tile b % q_tiles of doc tile b / q_tiles
  uint32_t block_stride;  // logical 32-doc block ub reads physical block ub * block_stride
  float inv_norm;
  // dense output (keys != null): keys[q * ld + u], u = logical doc
  uint32_t* keys;
  uint64_t ld;
  // filter output: (key, doc) with key <= thr[q * thr_stride] appended to row q
  const uint32_t* thr;
  uint64_t thr_stride;
  uint32_t* cnt;
  uint32_t cap;
  uint32_t* f_keys;
  uint32_t* f_ids;
  uint32_t* err;
};

__device__ __forceinline__ void rt_epi_bar() { asm volatile("bar.sync 1, %0;" ::"n"(kRtBuilders) : "memory"); }

__device__ __forceinline__ void rt_abort(RtSmem& S, uint32_t* err) {
  atomicExch(&S.abort, 1u);
  atomicOr(err, 1u);
}

__device__ __forceinline__ bool rt_aborted(const RtSmem& S) {
  return *reinterpret_cast<const volatile uint32_t*>(&S.abort) != 0;
}

template <int BITS>
__device__ __forceinline__ uint4 load_code_slice(const uint8_t* p, bool valid) {
  uint4 v = make_uint4(0, 0, 0, 0);
  if (valid) {
    if (BITS == 4) {
      v = __ldg(reinterpret_cast<const uint4*>(p));
    } else if (BITS == 2) {
      const uint2 u = __ldg(reinterpret_cast<const uint2*>(p));
      v.x = u.x;
      v.y = u.y;
    } else {
      v.x = __ldg(reinterpret_cast<const uint32_t*>(p));
    }
  }
  return v;
}

template <int BITS>
__global__ void __launch_bounds__(kRtThreads, 1)
    rank_tc_kernel(const __grid_constant__ CUtensorMap q_map, const RtArgs a) {
  extern __shared__ uint8_t smem_raw[];
  RtSmem& S = *reinterpret_cast<RtSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const uint32_t nt = a.nt;
  // query tiles vary fastest over the linear grid, so the CTAs of one doc tile
  // run together and its codes cross HBM once (the others read them from L2)
  const uint64_t dtile = blockIdx.x / a.q_tiles;
  const uint64_t r0 = (uint64_t)(blockIdx.x % a.q_tiles) * nt;  // first B row of the tile
  const uint64_t qb = r0 / 2;                     // first query of the tile
  const uint32_t nqt = (uint32_t)((a.nq - qb) < nt / 2 ? (a.nq - qb) : nt / 2);
  const uint32_t n_kb = a.dim / 64;
  const uint64_t n_blocks = (a.n + 31) / 32;
  const bool dense = a.keys != nullptr;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                 "r"(kRtTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 32) {
    for (int s = 0; s < kRtStages; s++) {
      mbar_init(&S.full_a[s], kRtBuilders / 32);
      mbar_init(&S.full_b[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    mbar_init(&S.acc_full, 1);
    S.abort = 0;
    S.epi_ok = 1;
    S.seg_full = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (uint32_t i = t; i < kRtMaxQ; i += kRtThreads) {
    S.thr[i] = (!dense && i < nqt) ? a.thr[(qb + i) * a.thr_stride] : 0u;
    S.cnt[i] = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S.tmem;

  if (warp == 0) {
    if (lane == 0) {
      const uint32_t b_bytes = nt * kRtKBytes;
      uint32_t issued = 0;
      for (uint32_t kb = 0; kb < n_kb; kb++) {
        const uint32_t s = kb % kRtStages, it = kb / kRtStages;
        if (rt_aborted(S)) break;
        if (kb >= kRtStages && !mbar_wait(&S.empty[s], (it - 1) & 1)) {
          rt_abort(S, a.err);
          break;
        }
        mbar_expect_tx(&S.full_b[s], b_bytes);
        tma_load_2d(S.b[s], &q_map, (int)(kb * 64), (int)r0, &S.full_b[s]);
        issued = kb + 1;
      }
      for (uint32_t kb = issued > kRtStages ? issued - kRtStages : 0; kb < issued; kb++)
        mbar_wait(&S.full_b[kb % kRtStages], (kb / kRtStages) & 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // D f32, A/B bf16, both K-major, N = nt, M = 128
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((nt >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
      uint32_t done = 0;
      for (uint32_t kb = 0; kb < n_kb; kb++) {
        const uint32_t s = kb % kRtStages, it = kb / kRtStages;
        if (rt_aborted(S)) break;
        if (!mbar_wait(&S.full_b[s], it & 1) || !mbar_wait(&S.full_a[s], it & 1)) {
          rt_abort(S, a.err);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_u32(S.a[s]), b0 = smem_u32(S.b[s]);
#pragma unroll
        for (uint32_t j = 0; j < 4; j++) {
          const uint64_t bd = sw128_desc(b0 + 32 * j);
          const uint32_t acc = (kb | j) != 0;
          mma_f16(tmem, sw128_desc(a0 + 32 * j), bd, idesc, acc);
          mma_f16(tmem + kRtAcc1Col, sw128_desc(a0 + kRtAHalf + 32 * j), bd, idesc, acc);
        }
        mma_commit(&S.empty[s]);
        done = kb + 1;
      }
      if (done == n_kb && !rt_aborted(S)) {
        mma_commit(&S.acc_full);
        mbar_wait(&S.acc_full, 0);
      } else if (done > 0) {
        mbar_wait(&S.empty[(done - 1) % kRtStages], ((done - 1) / kRtStages) & 1);
      }
    }
  } else {
    // ---- A builders: row r (doc within the tile), coordinates 32 hc .. 32 hc + 31 of each K-block
    const uint32_t bt = (uint32_t)t - 64;
    const uint32_t r = bt & 255, hc = bt >> 8;
    {
      uint32_t t0, t1;
      nibble_table<BITS>((uint32_t)lane, t0, t1);
      const uint64_t pb = (dtile * 8 + (r >> 5)) * a.block_stride;
      const uint64_t doc = pb * 32 + (r & 31);
      const bool valid = pb < n_blocks && doc < a.n;
      // this thread's 4 * BITS code bytes of each K-block (8 * BITS bytes per K-block row)
      const uint8_t* rc = a.codes + (valid ? doc : 0) * (uint64_t)a.bpv + hc * 4 * BITS;
      const uint32_t a_row = smem_u32(S.a[0]) + (r >> 7) * kRtAHalf + ((r & 127) >> 3) * 1024 + (r & 7) * 128;
      uint32_t dst[4];
#pragma unroll
      for (uint32_t c = 0; c < 4; c++) dst[c] = a_row + (((4 * hc + c) ^ (r & 7)) << 4);
      uint32_t s = 0, par = 0, base = 0;
      bool ok = true;
      uint4 nxt = load_code_slice<BITS>(rc, valid);
      for (uint32_t kb = 0; kb < n_kb && ok; kb++) {
        const uint4 cw = nxt;
        if (kb + 1 < n_kb) nxt = load_code_slice<BITS>(rc + (uint64_t)(kb + 1) * 8 * BITS, valid);
        if (kb >= (uint32_t)kRtStages) {
          if (lane == 0) ok = mbar_wait(&S.empty[s], par ^ 1);
          ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
          if (!ok) {
            if (lane == 0) rt_abort(S, a.err);
            break;
          }
          __syncwarp();
        }
        const uint32_t w[4] = {cw.x, cw.y, cw.z, cw.w};
#pragma unroll
        for (uint32_t c = 0; c < 4; c++) {  // 16-byte chunk c = coordinates 8c .. 8c+7
          uint32_t o[4];
          if (BITS == 2) {  // 4 nibbles (2 codes each) per chunk, 2 chunks per word
#pragma unroll
            for (int i = 0; i < 4; i++) o[i] = __shfl_sync(0xFFFFFFFFu, t0, nib(w[c >> 1], 4 * (c & 1) + i));
          } else if (BITS == 1) {  // 2 nibbles (4 codes each) per chunk
#pragma unroll
            for (int i = 0; i < 2; i++) {
              const uint32_t v = nib(w[0], 2 * c + i);
              o[2 * i] = __shfl_sync(0xFFFFFFFFu, t0, v);
              o[2 * i + 1] = __shfl_sync(0xFFFFFFFFu, t1, v);
            }
          } else {  // 8 nibbles (1 code each) per chunk: word c
#pragma unroll
            for (int i = 0; i < 4; i++)
              o[i] = __shfl_sync(0xFFFFFFFFu, t0, nib(w[c], 2 * i)) |
                     (__shfl_sync(0xFFFFFFFFu, t0, nib(w[c], 2 * i + 1)) << 16);
          }
          st_shared_v4(dst[c] + base, o[0], o[1], o[2], o[3]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&S.full_a[s]);
        base += kRtAStage;
        if (++s == kRtStages) {
          s = 0;
          base = 0;
          par ^= 1;
        }
      }
    }

    // ---- epilogue
    bool ready = false;
    if (lane == 0) {
      const uint32_t addr = smem_u32(&S.acc_full);
      uint64_t t0 = 0;
      for (uint32_t it = 0; it < kWaitLimit && !rt_aborted(S); it++) {
        if (mbar_try(addr, 0)) {
          ready = true;
          break;
        }
        if ((it & 255) == 255) {
          const uint64_t now = global_ns();
          if (!t0)
            t0 = now;
          else if (now - t0 > kWaitNs)
            break;
        }
      }
      if (!ready && !rt_aborted(S)) rt_abort(S, a.err);
    }
    ready = __shfl_sync(0xFFFFFFFFu, ready, 0);
    __syncwarp();
    if (!ready || rt_aborted(S)) atomicExch(&S.epi_ok, 0u);
    rt_epi_bar();
    ready = *reinterpret_cast<volatile uint32_t*>(&S.epi_ok) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ready) {
      const uint32_t eg = (uint32_t)(warp - 2) >> 2;
      const uint32_t h = eg & 1, c0 = (eg >> 1) * 32, lq = (uint32_t)warp & 3;
      const uint32_t row = h * 128 + lq * 32 + lane;
      const uint64_t pb = (dtile * 8 + (row >> 5)) * a.block_stride;
      const uint64_t doc = pb * 32 + lane;
      const uint64_t u = dtile * kRtM + row;
      const bool valid = pb < n_blocks && doc < a.n;
      const uint32_t taddr = tmem + ((lq * 32) << 16) + h * kRtAcc1Col;
      // filter list segment of this warp in the dead A stages
      uint2* list = reinterpret_cast<uint2*>(&S.a[0][0]) + (uint32_t)(warp - 2) * kRtSegCap;
      uint32_t wcount = 0;
      uint32_t lt;
      asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
      for (uint32_t cb = c0; cb < nt; cb += 64) {
        uint32_t v[32];
        __syncwarp();
        tmem_ld32(taddr + cb, v);
        uint32_t key[16];
#pragma unroll
        for (uint32_t p = 0; p < 16; p++)
          key[p] = desc_key(__fmul_rn(__fadd_rn(__uint_as_float(v[2 * p]), __uint_as_float(v[2 * p + 1])), a.inv_norm));
        if (dense) {
          if (valid) {
#pragma unroll
            for (uint32_t p = 0; p < 16; p++) {
              const uint64_t q = qb + cb / 2 + p;
              if (q < a.nq) a.keys[q * a.ld + u] = key[p];
            }
          }
          continue;
        }
        // filter: mask of the 16 queries this lane's doc passes, then ballot-ranked appends
        uint32_t hm = 0;
#pragma unroll
        for (uint32_t p = 0; p < 16; p++) {
          const uint32_t qi = cb / 2 + p;
          hm |= (uint32_t)(qi < nqt && key[p] <= S.thr[qi]) << p;
        }
        if (!valid) hm = 0;
        while (__any_sync(0xFFFFFFFFu, hm != 0)) {
          const bool has = hm != 0;
          const uint32_t p = has ? (uint32_t)(__ffs(hm) - 1) : 0u;
          const uint32_t bal = __ballot_sync(0xFFFFFFFFu, has);
          const uint32_t pos = wcount + __popc(bal & lt);
          if (has && pos < kRtSegCap) {
            uint32_t kk = key[0];
#pragma unroll
            for (uint32_t pp = 1; pp < 16; pp++) kk = pp == p ? key[pp] : kk;
            list[pos] = make_uint2(kk, (cb / 2 + p) | (row << 16));
          }
          wcount += __popc(bal);
          hm &= hm - 1;
        }
      }
      if (!dense) {
        const uint32_t total = wcount < kRtSegCap ? wcount : kRtSegCap;
        if (wcount > kRtSegCap && lane == 0) atomicExch(&S.seg_full, 1u);
        __syncwarp();
        for (uint32_t e = lane; e < total; e += 32) {
          const uint32_t y = list[e].y;
          list[e].y = y | (atom_add_shared(&S.cnt[y & 255], 1u) << 8);  // slot < 256
        }
        rt_epi_bar();
        const uint32_t i = (uint32_t)t - 64;
        if (i < nqt) {
          if (S.seg_full)  // some kept doc did not fit: bit 31 makes the count exceed any cap
            atomicOr(&a.cnt[qb + i], 0x80000000u);
          else if (S.cnt[i])
            S.base[i] = atomicAdd(&a.cnt[qb + i], S.cnt[i]);
        }
        rt_epi_bar();
        for (uint32_t e = lane; e < total; e += 32) {
          const uint2 en = list[e];
          const uint32_t q = en.y & 255, li = (en.y >> 8) & 255, rw = en.y >> 16;
          const uint32_t pos = S.base[q] + li;
          if (pos < a.cap) {
            a.f_keys[(qb + q) * a.cap + pos] = en.x;
            const uint64_t rpb = (dtile * 8 + (rw >> 5)) * a.block_stride;
            a.f_ids[(qb + q) * a.cap + pos] = (uint32_t)(rpb * 32 + (rw & 31));
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kRtTmemCols) : "memory");
}

// q_unit rows -> [hi; lo] bf16 rows (row 2i = hi of query i) and |q|_1.
__global__ void split_queries_kernel(const float* __restrict__ qu, uint64_t nq, uint32_t dim,
                                     __nv_bfloat16* __restrict__ out, float* __restrict__ l1) {
  __shared__ float part[32];
  const uint64_t i = blockIdx.x;
  const float* q = qu + i * dim;
  float s = 0.0f;
  for (uint32_t j = threadIdx.x; j < dim; j += blockDim.x) {
    const float x = q[j];
    const __nv_bfloat16 hi = __float2bfloat16_rn(x);
    const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));  // x - hi is exact in f32
    out[(2 * i) * dim + j] = hi;
    out[(2 * i + 1) * dim + j] = lo;
    s += fabsf(x);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float tot = 0.0f;
    for (uint32_t w = 0; w < blockDim.x / 32; w++) tot += part[w];
    l1[i] = tot * 1.0001f;  // covers the f32 rounding of the sum itself
  }
}

// Margin test of the split-BF16 candidates: flag |= 1 when a query's kp-th
// best split score is not below its k-th best minus twice the error bound.
__global__ void split_margin_kernel(const uint32_t* __restrict__ sel_keys, uint64_t nq, uint32_t kp, uint32_t k,
                                    const float* __restrict__ l1, float bound_per_l1, uint32_t* __restrict__ flag) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  const float tk = desc_key_to_float(sel_keys[i * kp + (k - 1)]);
  const float last = desc_key_to_float(sel_keys[i * kp + (kp - 1)]);
  const float eps = l1[i] * bound_per_l1;
  // written so that NaN anywhere fails the test
  if (!(last < tk - 2.0f * eps - 4.0f * fabsf(tk) * 1.1920929e-7f)) atomicOr(flag, 1u);
}

}  // namespace

bool rank_tc_eligible(uint32_t dim, uint32_t bits) {
  return dim % 64 == 0 && dim >= 64 && (bits == 1 || bits == 2 || bits == 4);
}

float split_error_bound(uint32_t dim, uint32_t bits, float inv_norm) {
  // |split score - exact| <= inv_norm * c_max * |q|_1 * (2 dim u + 2^-16) * 1.05 (u = 2^-24): f32
  // accumulation of 2 dim exact products in any order, plus |q - hi - lo| <= 2^-16 |q|
  const double cmax = ((double)(1u << bits) - 1.0) * 0.5;
  return (float)((double)inv_norm * cmax * (2.0 * dim * 5.9604644775390625e-8 + 1.52587890625e-5) * 1.05);
}

void launch_split_queries(const float* q_unit, uint64_t nq, uint32_t dim, void* out_bf16, float* l1,
                          cudaStream_t stream) {
  if (!nq) return;
  split_queries_kernel<<<(unsigned)nq, 256, 0, stream>>>(q_unit, nq, dim, (__nv_bfloat16*)out_bf16, l1);
  launched();
}

void launch_split_margin(const uint32_t* sel_keys, uint64_t nq, uint32_t kp, uint32_t k, const float* l1,
                         float bound_per_l1, uint32_t* flag, cudaStream_t stream) {
  if (!nq) return;
  split_margin_kernel<<<(unsigned)((nq + 255) / 256), 256, 0, stream>>>(sel_keys, nq, kp, k, l1, bound_per_l1, flag);
  launched();
}

static void launch_rank_tc(RtArgs a, uint32_t bits, const void* q_split, uint32_t q_per_tile, cudaStream_t stream) {
  if (!a.n || !a.nq) return;
  if (!rank_tc_eligible(a.dim, bits)) throw std::invalid_argument("rank tensor-core scan: dim must be a multiple of 64");
  a.bpv = a.dim * bits / 8;
  if (!a.block_stride) a.block_stride = 1;
  if (!a.keys && a.block_stride != 1) throw std::invalid_argument("rank tensor-core scan: filter needs stride 1");
  uint32_t qt = q_per_tile ? q_per_tile : 128;  // queries per tile: 8..128, multiple of 8
  if (qt > 128) qt = 128;
  if ((uint64_t)qt > a.nq) qt = (uint32_t)a.nq;
  qt = (qt + 7) / 8 * 8;
  a.nt = 2 * qt;
  CUtensorMap map;
  cuuint64_t gdim[2] = {(cuuint64_t)a.dim, (cuuint64_t)(2 * a.nq)};
  cuuint64_t gstride[1] = {(cuuint64_t)a.dim * 2};
  cuuint32_t box[2] = {64, a.nt};
  cuuint32_t estride[2] = {1, 1};
  CUresult rc = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(q_split), gdim, gstride,
                            box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rc != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed for the split query matrix");
  const size_t smem = sizeof(RtSmem) + 1024;
  const uint64_t n_blocks = (a.n + 31) / 32;
  const uint64_t logical_blocks = (n_blocks + a.block_stride - 1) / a.block_stride;
  const uint64_t doc_tiles = (logical_blocks + 7) / 8;
  const uint64_t q_tiles = (2 * a.nq + a.nt - 1) / a.nt;
  if (q_tiles * doc_tiles > 0x7FFFFFFFull || a.n >= (1ull << 32))
    throw std::invalid_argument("rank tensor-core scan: grid too large; split the query batch");
  a.q_tiles = (uint32_t)q_tiles;
  dim3 grid((unsigned)(q_tiles * doc_tiles));
#define OVB_RT(B)                                                                                              \
  do {                                                                                                         \
    allow_dynamic_smem(rank_tc_kernel<B>);                                                                    \
    rank_tc_kernel<B><<<grid, kRtThreads, smem, stream>>>(map, a);                                            \
  } while (0)
  if (bits == 1)
    OVB_RT(1);
  else if (bits == 2)
    OVB_RT(2);
  else
    OVB_RT(4);
#undef OVB_RT
  launched();
}

void launch_rank_scan_tc(const uint8_t* codes, uint64_t n, uint32_t dim, uint32_t bits, const void* q_split,
                         uint64_t nq, float inv_norm, uint32_t block_stride, uint32_t* keys, uint64_t ld,
                         uint32_t q_per_tile, uint32_t* err, cudaStream_t stream) {
  RtArgs a{};
  a.codes = codes;
  a.n = n;
  a.dim = dim;
  a.nq = nq;
  a.block_stride = block_stride;
  a.inv_norm = inv_norm;
  a.keys = keys;
  a.ld = ld;
  a.err = err;
  launch_rank_tc(a, bits, q_split, q_per_tile, stream);
}

void launch_rank_filter_tc(const uint8_t* codes, uint64_t n, uint32_t dim, uint32_t bits, const void* q_split,
                           uint64_t nq, float inv_norm, const uint32_t* thr, uint64_t thr_stride, uint32_t* cnt,
                           uint32_t cap, uint32_t* f_keys, uint32_t* f_ids, uint32_t q_per_tile, uint32_t* err,
                           cudaStream_t stream) {
  RtArgs a{};
  a.codes = codes;
  a.n = n;
  a.dim = dim;
  a.nq = nq;
  a.block_stride = 1;
  a.inv_norm = inv_norm;
  a.thr = thr;
  a.thr_stride = thr_stride;
  a.cnt = cnt;
  a.cap = cap;
  a.f_keys = f_keys;
  a.f_ids = f_ids;
  a.err = err;
  launch_rank_tc(a, bits, q_split, q_per_tile, stream);
}

}  // namespace ovb
