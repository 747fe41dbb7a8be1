// K3 on the 5th-generation tensor cores: FastScan b=2 scoring of many queries
// at once as an exact integer GEMM.
//
//   acc[doc][q] = sum_p LUT_q[p][nib_p(doc)] = sum_k onehot(doc)[k] * LUT_q[k],
//   k = 16 p + nibble  (K = pairs_pad * 16 = 8192 at dim 1024)
//
// A (docs x K) is the one-hot expansion of the nibble codes, built in shared
// memory by the CTA's threads; B (N = up to 256 queries x K) is the u8 LUT
// matrix, loaded by TMA; D (s32) accumulates in tensor memory with
// tcgen05.mma kind::i8 (u8 x u8).  A CTA owns 256 docs as two M=128
// accumulators (TMEM columns [0, N) and [256, 256 + N)), so every LUT byte it
// loads feeds 256 docs.  Both operands use the K-major 128-byte swizzled
// layout: row r of a 128-byte K-block at (r/8)*1024 + (r%8)*128, its 16-byte
// chunk c at ((c ^ r%8) * 16).  The sum is exact, so the scores
//   (bias + (acc as f32) * inv_q) * inv_norm
// equal the CUDA-core kernel's (and the reference's) bit for bit.
//
// Warp roles (576 threads):
//   warp 0, lane 0   TMA producer: LUT K-block -> stage s   (waits empty[s])
//   warp 1, lane 0   MMA issuer: 8 MMAs per K-block, commit -> empty[s]
//   warps 2..17      A builders, two threads per doc row, four 16-byte chunks
//                    each (wait empty[s], one arrive per warp on full_a[s]);
//                    afterwards the epilogue (TMEM -> keys)
// STAGES smem stages of (A 32 KiB + B 32 KiB) let the producer and builders run
// ahead of the tensor core.  Every wait is bounded: on timeout the kernel sets
// bit 0 of *err, stops issuing work, waits (bounded) for the copies and MMAs it
// issued, frees its tensor memory and returns.
//
// Epilogue modes:
//   dense   keys[q][u] = key32 for every logical doc u (the key matrix)
//   filter  only keys <= thr[q] are appended to row q of a capacity-`cap`
//           buffer (key, doc id) through an atomic counter; cnt[q] ends as the
//           number of qualifying docs even when it exceeds `cap`, or with bit
//           31 set when a tile kept more than its shared-memory list holds
//           (either way cnt[q] > cap and the caller redoes the query densely).
// Doc sampling: logical 32-doc block ub reads physical block ub * block_stride,
// so a stride > 1 scores an evenly spread sample of the index.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "ovb_common.cuh"
#include "ovb_kernels.h"
#include "tc_common.cuh"
#include "tc_scan.cuh"

namespace ovb {

namespace {

using namespace tc;
using namespace tcs;

constexpr int kTcThreads = 576;
constexpr int kTcBuilders = 512;  // warps 2..17
constexpr int kTcM = 256;         // docs per CTA (two M=128 accumulators)
constexpr int kTcMaxN = 256;
constexpr int kTcKBytes = 128;  // 8 pairs x 16 one-hot bytes per K-block
constexpr int kTcStages = 3;
constexpr uint32_t kAHalf = 128 * kTcKBytes;        // 16 KiB
constexpr uint32_t kAStage = kTcM * kTcKBytes;      // 32 KiB
constexpr uint32_t kBStage = kTcMaxN * kTcKBytes;   // 32 KiB
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kAcc1Col = 256;
// filter epilogue list (accumulator, q | slot << 8 | row << 16) in the dead A stages,
// one segment per epilogue warp
constexpr uint32_t kListCap = kTcStages * kAStage / 8;
constexpr uint32_t kSegCap = kListCap / (kTcBuilders / 32);

struct TcSmem {
  uint8_t a[kTcStages][kAStage];
  uint8_t b[kTcStages][kBStage];
  float bias[kTcMaxN];
  float invq[kTcMaxN];
  uint32_t thr[kTcMaxN];
  uint32_t amin[kTcMaxN];  // filter: smallest passing accumulator, or kExactCompare
  uint32_t tdoc[kTcMaxN];  // bitmap filter, tie level: last passing doc id
  uint32_t qpop[kTcMaxN];  // sign bitmaps: query popcounts
  uint64_t full_a[kTcStages];
  uint64_t full_b[kTcStages];
  uint64_t empty[kTcStages];
  uint64_t acc_full;
  uint32_t cnt[kTcMaxN];   // filter: kept docs per query in this tile
  uint32_t base[kTcMaxN];  // filter: the tile's first slot in each query row
  uint32_t epi_ok;
  uint32_t seg_full;   // filter: some warp's list segment overflowed
  uint32_t any_exact;  // filter: some query of the tile needs key compares
  uint32_t tmem;
  uint32_t abort;
};




// named barrier 1 over the builder / epilogue threads (warps 2..17)
__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, %0;" ::"n"(kTcBuilders) : "memory"); }

__device__ __forceinline__ void raise_abort(TcSmem& S, uint32_t* err) {
  atomicExch(&S.abort, 1u);
  atomicOr(err, 1u);
}

__device__ __forceinline__ bool aborted(const TcSmem& S) {
  return *reinterpret_cast<const volatile uint32_t*>(&S.abort) != 0;
}






template <int MODE>
__device__ __forceinline__ void tc_scan_body(const CUtensorMap& lut_map, const TcArgs& a) {
  extern __shared__ uint8_t smem_raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const uint64_t q0 = (uint64_t)blockIdx.y * a.nt;
  const uint32_t nt = a.nt;
  const uint32_t nqt = (uint32_t)((a.nq - q0) < nt ? (a.nq - q0) : nt);
  const uint64_t n_blocks = (a.n + 31) / 32;
  const uint32_t n_kb = a.n_kb;
  const bool dense = a.keys != nullptr;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 32) {
    for (int s = 0; s < kTcStages; s++) {
      mbar_init(&S.full_a[s], kTcBuilders / 32);  // one arrive per builder warp
      mbar_init(&S.full_b[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    mbar_init(&S.acc_full, 1);
    S.abort = 0;
    S.epi_ok = 1;
    S.seg_full = 0;
    S.any_exact = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (uint32_t i = t; i < nt; i += kTcThreads) {
    const bool v = i < nqt;
    S.bias[i] = (MODE == 0 && v) ? a.bias[q0 + i] : 0.0f;
    S.invq[i] = (MODE == 0 && v) ? a.invq[q0 + i] : 0.0f;
    S.thr[i] = (v && !dense) ? a.thr[(q0 + i) * a.thr_stride] : 0u;
    S.qpop[i] = (MODE == 1 && v && a.key_kind == 2) ? a.qpop[q0 + i] : 0u;
    if (MODE == 0)
      S.amin[i] = !v ? kNeverPasses
                     : dense ? kExactCompare
                             : filter_amin(S.bias[i], S.invq[i], a.inv_norm, S.thr[i], 255u * a.pairs_pad);
    else if (!v || dense)
      S.amin[i] = v ? 0u : kNeverPasses;
    else {
      // key <= thr  <=>  acc >= am.  With a tie bound, (key, doc) <= (thr, tdoc):
      // this tile's docs [first, first + 256) all pass the tie level, none do,
      // or the compare is per doc (kExactCompare, am kept in thr).
      const uint32_t am = bm_amin_q(a, S.qpop[i], S.thr[i]);
      S.amin[i] = am;
      if (a.thr_pos) {
        const uint32_t p = a.thr_pos[(q0 + i) * a.thr_stride];
        const uint64_t td = ((uint64_t)(p >> 5) * a.smp_stride) * 32 + (p & 31);
        const uint64_t first = (uint64_t)blockIdx.x * kTcM;
        S.tdoc[i] = (uint32_t)td;
        S.thr[i] = am;
        S.amin[i] = td >= first + kTcM - 1 ? am : td < first ? am + 1 : kExactCompare;
      }
    }
    S.cnt[i] = 0;
  }
  __syncthreads();  // barrier init and amin visible to every thread
  for (uint32_t i = t; i < nt; i += kTcThreads)
    if (S.amin[i] == kExactCompare) atomicOr(&S.any_exact, 1u);
  for (uint32_t i = nt + t; i < kTcMaxN; i += kTcThreads) S.amin[i] = kNeverPasses;
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S.tmem;

  if (warp == 0) {
    // ---- TMA producer --------------------------------------------------------
    if (lane == 0) {
      const uint32_t b_bytes = nt * kTcKBytes;
      uint32_t issued = 0;
      for (uint32_t kb = 0; kb < n_kb; kb++) {
        const uint32_t s = kb % kTcStages, it = kb / kTcStages;
        if (aborted(S)) break;
        if (kb >= kTcStages && !mbar_wait(&S.empty[s], (it - 1) & 1)) {
          raise_abort(S, a.err);
          break;
        }
        mbar_expect_tx(&S.full_b[s], b_bytes);
        tma_load_2d(S.b[s], &lut_map, (int)(kb * kTcKBytes), (int)q0, &S.full_b[s]);
        issued = kb + 1;
      }
      // every issued copy lands before the CTA exits (the latest phase of each
      // stage covers the earlier ones)
      for (uint32_t kb = issued > kTcStages ? issued - kTcStages : 0; kb < issued; kb++)
        mbar_wait(&S.full_b[kb % kTcStages], (kb / kTcStages) & 1);
    }
  } else if (warp == 1) {
    // ---- MMA issuer ----------------------------------------------------------
    if (lane == 0) {
      // D s32, A/B u8, both K-major, N = nt, M = 128
      const uint32_t idesc = (2u << 4) | ((nt >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
      uint32_t done = 0;
      for (uint32_t kb = 0; kb < n_kb; kb++) {
        const uint32_t s = kb % kTcStages, it = kb / kTcStages;
        if (aborted(S)) break;
        if (!mbar_wait(&S.full_b[s], it & 1) || !mbar_wait(&S.full_a[s], it & 1)) {
          raise_abort(S, a.err);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_u32(S.a[s]), b0 = smem_u32(S.b[s]);
#pragma unroll
        for (uint32_t j = 0; j < 4; j++) {
          const uint64_t bd = sw128_desc(b0 + 32 * j);
          const uint32_t acc = (kb | j) != 0;
          mma_i8(tmem, sw128_desc(a0 + 32 * j), bd, idesc, acc);
          mma_i8(tmem + kAcc1Col, sw128_desc(a0 + kAHalf + 32 * j), bd, idesc, acc);
        }
        mma_commit(&S.empty[s]);
        done = kb + 1;
      }
      // the issuer itself waits (bounded) for its last commit, which covers
      // every earlier MMA, so no MMA is in flight when the CTA frees TMEM
      if (done == n_kb && !aborted(S)) {
        mma_commit(&S.acc_full);
        mbar_wait(&S.acc_full, 0);
      } else if (done > 0) {
        mbar_wait(&S.empty[(done - 1) % kTcStages], ((done - 1) / kTcStages) & 1);
      }
    }
  } else {
    // ---- A builders: row r = doc (tile-local), chunks 4*hc .. 4*hc+3 ----------
    const uint32_t bt = (uint32_t)t - 64;
    const uint32_t r = bt & 255, hc = bt >> 8;
    if constexpr (MODE == 1) {
      // bitmap rows, bit j of word j/64 = coordinate j: thread hc expands word
      // 2 kb + hc (coordinates 64 hc .. 64 hc + 63 of K-block kb) to 0/1 bytes
      const uint64_t pb = ((uint64_t)blockIdx.x * 8 + (r >> 5)) * a.block_stride;
      const uint64_t doc = pb * 32 + (r & 31);
      const bool row_ok = pb < n_blocks && doc < a.n;
      const uint64_t* words = reinterpret_cast<const uint64_t*>(a.blocks) + (row_ok ? doc : 0) * (uint64_t)a.qpv;
      const uint32_t a_row = smem_u32(S.a[0]) + (r >> 7) * kAHalf + ((r & 127) >> 3) * 1024 + (r & 7) * 128;
      uint32_t dst[4];
#pragma unroll
      for (uint32_t c = 0; c < 4; c++) dst[c] = a_row + (((4 * hc + c) ^ (r & 7)) << 4);
      auto word_at = [&](uint32_t kb) -> uint64_t {
        const uint32_t wi = 2 * kb + hc;
        return (row_ok && wi < a.qpv) ? __ldg(words + wi) : 0ull;
      };
      uint32_t s = 0, par = 0, base = 0;
      bool ok = true;
      // four K-blocks of words in flight (the tile's first loads are the
      // latency that is not hidden)
      uint64_t w0 = word_at(0), w1 = word_at(1), w2 = word_at(2), w3 = word_at(3);
      for (uint32_t kb = 0; kb < n_kb && ok; kb++) {
        const uint64_t wd = w0;
        w0 = w1;
        w1 = w2;
        w2 = w3;
        w3 = kb + 4 < n_kb ? word_at(kb + 4) : 0ull;
        if (kb >= (uint32_t)kTcStages) {
          if (lane == 0) ok = mbar_wait(&S.empty[s], par ^ 1);
          ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
          if (!ok) {
            if (lane == 0) raise_abort(S, a.err);
            break;
          }
          __syncwarp();
        }
#pragma unroll
        for (uint32_t c = 0; c < 4; c++) {  // 16 coordinates per 16-byte chunk
          const uint32_t h = (uint32_t)(wd >> (16 * c));
          uint32_t o[4];
#pragma unroll
          for (uint32_t i = 0; i < 4; i++)  // 4 bits -> 4 bytes (the shifted copies never overlap)
            o[i] = (((h >> (4 * i)) & 15u) * 0x00204081u) & 0x01010101u;
          st_shared_v4(dst[c] + base, o[0], o[1], o[2], o[3]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&S.full_a[s]);
        base += kAStage;
        if (++s == kTcStages) {
          s = 0;
          base = 0;
          par ^= 1;
        }
      }
    } else
    {
      const uint64_t pb = ((uint64_t)blockIdx.x * 8 + (r >> 5)) * a.block_stride;
      const bool row_valid = pb < n_blocks;
      const uint8_t* row_codes = a.blocks + pb * (uint64_t)a.pairs_pad * 16 + (uint64_t)(r & 31) * 16;
      // shared-space addresses of this thread's four 16-byte chunks in stage 0
      const uint32_t a_row = smem_u32(S.a[0]) + (r >> 7) * kAHalf + ((r & 127) >> 3) * 1024 + (r & 7) * 128;
      uint32_t dst[4];
#pragma unroll
      for (uint32_t c = 0; c < 4; c++) dst[c] = a_row + (((4 * hc + c) ^ (r & 7)) << 4);
      // one 16-byte code load covers a 32-pair group = 4 K-blocks
      const uint32_t n_groups = n_kb / 4;
      uint4 next = row_valid ? load_codes(row_codes) : make_uint4(0, 0, 0, 0);
      uint32_t s = 0, par = 0, base = 0;  // stage of kb, parity of kb / kTcStages, stage offset
      bool ok = true;
      for (uint32_t g = 0; g < n_groups && ok; g++) {
        const uint4 chunk = next;
        if (row_valid && g + 1 < n_groups) next = load_codes(row_codes + (uint64_t)(g + 1) * 512);
#pragma unroll
        for (uint32_t j = 0; j < 4; j++) {
          // warp-uniform control flow: lane 0 waits for the stage, the warp
          // follows its verdict
          if (4 * g + j >= (uint32_t)kTcStages) {
            if (lane == 0) ok = mbar_wait(&S.empty[s], par ^ 1);
            ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
            if (!ok) {
              if (lane == 0) raise_abort(S, a.err);
              break;
            }
            __syncwarp();
          }
          const uint32_t w = (j == 0 ? chunk.x : j == 1 ? chunk.y : j == 2 ? chunk.z : chunk.w) >> (16 * hc);
#pragma unroll
          for (uint32_t c = 0; c < 4; c++) {
            const uint32_t sh = c == 0 ? (w << 3) & 0x78u : (w >> (4 * c - 3)) & 0x78u;  // 8 * nibble
            st_shared_v4(dst[c] + base, shl1(sh), shl1(sh - 32), shl1(sh - 64), shl1(sh - 96));
          }
          // each lane makes its rows visible to the tensor core's (async) proxy;
          // the warp barrier orders all lanes before lane 0's release-arrive
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(&S.full_a[s]);
          base += kAStage;
          if (++s == kTcStages) {
            s = 0;
            base = 0;
            par ^= 1;
          }
        }
      }
    }

    // ---- epilogue: TMEM lane quarter (warp % 4), accumulator half ------------
    bool ready = false;
    if (lane == 0) {
      const uint32_t addr = smem_u32(&S.acc_full);
      uint64_t t0 = 0;
      for (uint32_t it = 0; it < kWaitLimit && !aborted(S); it++) {
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
      if (!ready && !aborted(S)) raise_abort(S, a.err);
    }
    ready = __shfl_sync(0xFFFFFFFFu, ready, 0);
    __syncwarp();
    // one decision for all epilogue threads (they share named barrier 1)
    if (!ready || aborted(S)) atomicExch(&S.epi_ok, 0u);
    epi_bar();
    ready = *reinterpret_cast<volatile uint32_t*>(&S.epi_ok) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ready) {
      // warps 2..17: TMEM lane quarter warp % 4 (hardware rule), accumulator
      // half h, and every other 32-column chunk starting at c0
      const uint32_t eg = (uint32_t)(warp - 2) >> 2;
      const uint32_t h = eg & 1, c0 = (eg >> 1) * 32, lq = (uint32_t)warp & 3;
      const uint32_t row = h * 128 + lq * 32 + lane;
      const uint64_t pb = ((uint64_t)blockIdx.x * 8 + (row >> 5)) * a.block_stride;
      const uint64_t doc = pb * 32 + lane;
      const uint64_t u = (uint64_t)blockIdx.x * kTcM + row;
      const bool valid = pb < n_blocks && doc < a.n;
      const uint32_t dpop = (MODE == 1 && a.key_kind == 2) ? row_popcount(a, doc, valid) : 0u;
      const uint32_t taddr = tmem + ((lq * 32) << 16) + h * kAcc1Col;
      const bool any_exact = S.any_exact != 0;
      // filter list: the A stages are dead once acc_full has fired; each warp
      // appends to its own segment with a register counter (ballot ranks), so
      // only the per-query slot counters see shared-memory atomics
      uint2* list = reinterpret_cast<uint2*>(&S.a[0][0]) + (uint32_t)(warp - 2) * kSegCap;
      uint32_t wcount = 0;
      uint32_t lt;
      asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
      for (uint32_t cb = c0; cb < nt; cb += 64) {
        uint32_t v[32];
        __syncwarp();
        tmem_ld32(taddr + cb, v);
        if (MODE == 1 && a.key_kind == 2) {
#pragma unroll
          for (uint32_t j = 0; j < 32; j++) v[j] = ham_y(v[j], dpop);
        }
        if (dense) {
#pragma unroll
          for (uint32_t j = 0; j < 32; j++) {
            const uint32_t q = cb + j;
            if (valid && q < nqt)
              a.keys[(q0 + q) * a.ld + u] =
                  MODE == 0 ? desc_key(tc_score(v[j], S.bias[q], S.invq[q], a.inv_norm)) : bm_key_q(a, S.qpop[q], v[j]);
          }
          continue;
        }
        // filter: each lane (row) builds the mask of the 32 queries its doc
        // passes (amin is kNeverPasses past nqt); kept docs are rare (m << n),
        // so the appends run once per set bit of the busiest lane's mask
        uint32_t hm = 0;
        if (!any_exact) {  // the common case: accumulator compares only
#pragma unroll
          for (uint32_t j = 0; j < 32; j += 4) {
            const uint4 am = *reinterpret_cast<const uint4*>(&S.amin[cb + j]);
            hm |= ((uint32_t)(v[j] >= am.x) << j) | ((uint32_t)(v[j + 1] >= am.y) << (j + 1)) |
                  ((uint32_t)(v[j + 2] >= am.z) << (j + 2)) | ((uint32_t)(v[j + 3] >= am.w) << (j + 3));
          }
        } else {
#pragma unroll
          for (uint32_t j = 0; j < 32; j++) {
            const uint32_t q = cb + j;  // < kTcMaxN; same q in every lane
            const uint32_t am = S.amin[q];
            bool pass;
            if (am != kExactCompare)
              pass = v[j] >= am;
            else if (MODE == 0)
              pass = desc_key(tc_score(v[j], S.bias[q], S.invq[q], a.inv_norm)) <= S.thr[q];
            else
              pass = v[j] > S.thr[q] || (v[j] == S.thr[q] && doc <= S.tdoc[q]);
            hm |= (uint32_t)pass << j;
          }
        }
        if (!valid) hm = 0;
        // appends at ballot-prefix offsets of the warp's segment; no atomics
        while (__any_sync(0xFFFFFFFFu, hm != 0)) {
          const bool has = hm != 0;
          const uint32_t j = has ? (uint32_t)(__ffs(hm) - 1) : 0u;
          const uint32_t bal = __ballot_sync(0xFFFFFFFFu, has);
          const uint32_t e = wcount + __popc(bal & lt);
          if (has && e < kSegCap) {
            uint32_t acc = v[0];
#pragma unroll
            for (uint32_t jj = 1; jj < 32; jj++) acc = jj == j ? v[jj] : acc;
            list[e] = make_uint2(acc, (cb + j) | (row << 16));
          }
          wcount += __popc(bal);
          hm &= hm - 1;
        }
      }
      if (!dense) {
        // slots within each query's share of the tile (lane-parallel atomics),
        // one global atomic per query per tile, then each warp writes its segment
        const uint32_t total = wcount < kSegCap ? wcount : kSegCap;
        if (wcount > kSegCap && lane == 0) atomicExch(&S.seg_full, 1u);
        __syncwarp();  // entries were appended by every lane of the warp
        for (uint32_t e = lane; e < total; e += 32) {
          const uint32_t y = list[e].y;
          list[e].y = y | (atom_add_shared(&S.cnt[y & 255], 1u) << 8);  // slot < 256
        }
        epi_bar();
        const uint32_t i = (uint32_t)t - 64;
        if (i < nqt) {
          if (S.seg_full)  // some kept doc did not fit: mark every query (bit 31 > cap)
            atomicOr(&a.cnt[q0 + i], 0x80000000u);  // so the chunk is redone densely
          else if (S.cnt[i])
            S.base[i] = atomicAdd(&a.cnt[q0 + i], S.cnt[i]);
        }
        epi_bar();
        for (uint32_t e = lane; e < total; e += 32) {
          const uint2 en = list[e];  // (accumulator, q | slot << 8 | row << 16)
          const uint32_t q = en.y & 255, li = (en.y >> 8) & 255, rw = en.y >> 16;
          const uint32_t pos = S.base[q] + li;
          if (pos < a.cap) {
            a.f_keys[(q0 + q) * a.cap + pos] =
                MODE == 0 ? desc_key(tc_score(en.x, S.bias[q], S.invq[q], a.inv_norm)) : bm_key_q(a, S.qpop[q], en.x);
            const uint64_t rpb = ((uint64_t)blockIdx.x * 8 + (rw >> 5)) * a.block_stride;
            a.f_ids[(q0 + q) * a.cap + pos] = (uint32_t)(rpb * 32 + (rw & 31));
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

__global__ void __launch_bounds__(kTcThreads, 1)
    fastscan_tc_kernel(const __grid_constant__ CUtensorMap lut_map, const TcArgs a) {
  tc_scan_body<0>(lut_map, a);
}

__global__ void __launch_bounds__(kTcThreads, 1)
    bitmap_tc_kernel(const __grid_constant__ CUtensorMap q_map, const TcArgs a) {
  tc_scan_body<1>(q_map, a);
}

// popcount of each query's qpv words
__global__ void query_popcount_kernel(const uint64_t* __restrict__ qbits, uint64_t nq, uint32_t qpv,
                                      uint32_t* __restrict__ out) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  uint32_t c = 0;
  for (uint32_t i = 0; i < qpv; i++) c += __popcll(qbits[q * qpv + i]);
  out[q] = c;
}

// query bits (qpv u64 words per query) -> 0/1 bytes, row_bytes per query
__global__ void expand_query_bits_kernel(const uint64_t* __restrict__ qbits, uint64_t nq, uint32_t qpv,
                                         uint32_t row_bytes, uint8_t* __restrict__ out) {
  const uint64_t total = nq * (uint64_t)row_bytes;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t q = t / row_bytes;
    const uint32_t j = (uint32_t)(t % row_bytes);
    out[t] = (j / 64 < qpv) ? (uint8_t)((qbits[q * qpv + j / 64] >> (j % 64)) & 1ull) : 0;
  }
}

// query bits -> packed e2m1 nibbles (byte j: coordinate 2 j in the low nibble,
// 2 j + 1 in the high one; 0b0010 = 1.0 where the bit is set), row_bytes per query
__global__ void expand_query_nibbles_kernel(const uint64_t* __restrict__ qbits, uint64_t nq, uint32_t qpv,
                                            uint32_t row_bytes, uint8_t* __restrict__ out) {
  const uint64_t total = nq * (uint64_t)row_bytes;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t q = t / row_bytes;
    const uint32_t j = (uint32_t)(t % row_bytes);
    uint32_t v = 0;
    if (j / 32 < qpv) {
      const uint32_t two = (uint32_t)(qbits[q * qpv + j / 32] >> ((2 * j) % 64)) & 3u;
      v = ((two & 1u) ? 0x02u : 0u) | ((two & 2u) ? 0x20u : 0u);
    }
    out[t] = (uint8_t)v;
  }
}

__global__ void filter_check_kernel(const uint32_t* __restrict__ cnt, uint64_t nq, uint32_t need, uint32_t cap,
                                    uint32_t* __restrict__ flag) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nq) {
    const uint32_t c = cnt[i];
    if (c < need || c > cap) atomicOr(flag, 1u);
  }
}


template <int MODE>
void launch_tc(TcArgs a, const uint8_t* b_rows, cudaStream_t stream) {
  if (!a.n || !a.nq) return;
  TcForm form = tc_form(MODE);
  if (form == TcForm::kPersist && !a.keys) {
    // the persistent one-CTA form holds fewer kept entries per warp and tile
    // than this form's (the dead A stages): use it when twice the expected
    // share of a warp (32 docs x 128 queries) fits
    const double per_warp = a.expect_kept ? (double)a.expect_kept * 32.0 / (double)a.n : 1e9;
    if (2.0 * per_warp * 128.0 > (double)tc_persist_seg_cap()) form = TcForm::kTile;
  }
  if (form != TcForm::kTile) {
    launch_tc_pair<MODE>(a, b_rows, stream, form == TcForm::kPair);
    return;
  }
  const char* what = MODE == 0 ? "FastScan tensor-core scan" : "bitmap tensor-core scan";
  const uint64_t k_bytes = (uint64_t)a.n_kb * kTcKBytes;
  if (!a.n_kb || (MODE == 0 && a.n_kb % 4)) throw std::invalid_argument(std::string(what) + ": bad K extent");
  // N per tile: a multiple of 16 in [16, 256]
  a.nt = a.nq >= kTcMaxN ? kTcMaxN : (uint32_t)((a.nq + 15) / 16 * 16);
  CUtensorMap map;
  cuuint64_t gdim[2] = {(cuuint64_t)k_bytes, (cuuint64_t)a.nq};
  cuuint64_t gstride[1] = {(cuuint64_t)k_bytes};
  cuuint32_t box[2] = {(cuuint32_t)kTcKBytes, (cuuint32_t)a.nt};
  cuuint32_t estride[2] = {1, 1};
  CUresult rc = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)b_rows, gdim, gstride, box, estride,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rc != CUDA_SUCCESS) throw CudaError(std::string("cuTensorMapEncodeTiled failed: ") + what);
  if (MODE == 0 && 255ull * a.pairs_pad >= (1ull << 23))  // acc_to_float range
    throw std::invalid_argument(std::string(what) + ": dimension too large");
  if (MODE == 1 && (64ull * a.qpv >= (1ull << 24) || 2ull * a.n_kb < a.qpv))
    throw std::invalid_argument(std::string(what) + ": row too long");
  if (!a.keys && a.block_stride != 1) throw std::invalid_argument(std::string(what) + ": filter needs stride 1");
  auto kernel = MODE == 0 ? fastscan_tc_kernel : bitmap_tc_kernel;
  const size_t smem = sizeof(TcSmem) + 1024;
  OVB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const uint64_t n_blocks = (a.n + 31) / 32;
  const uint64_t logical_blocks = (n_blocks + a.block_stride - 1) / a.block_stride;
  const uint64_t doc_tiles = (logical_blocks + 7) / 8;
  const uint64_t q_tiles = (a.nq + a.nt - 1) / a.nt;
  if (q_tiles > 65535 || doc_tiles > 0x7FFFFFFF || a.n >= (1ull << 32))
    throw std::invalid_argument(std::string(what) + ": grid too large; split the query batch");
  dim3 grid((unsigned)doc_tiles, (unsigned)q_tiles);
  kernel<<<grid, kTcThreads, smem, stream>>>(map, a);
  launched();
}

}  // namespace

uint64_t fastscan_tc_sample_docs(uint64_t n, uint32_t block_stride) {
  const uint64_t n_blocks = (n + 31) / 32;
  if (!n_blocks) return 0;
  const uint64_t sampled = (n_blocks + block_stride - 1) / block_stride;
  const uint64_t last = (sampled - 1) * block_stride;  // the only block that can be partial
  return (sampled - 1) * 32 + (last == n_blocks - 1 ? n - last * 32 : 32);
}

void launch_fastscan_scan_tc(const uint8_t* blocks, uint64_t n, uint32_t pairs_pad, const uint8_t* lut,
                             const float* bias_sum, const float* inv_q, float inv_norm, uint64_t nq,
                             uint32_t block_stride, uint32_t* keys, uint64_t ld, uint32_t* err,
                             cudaStream_t stream) {
  TcArgs a{};
  a.blocks = blocks;
  a.n = n;
  a.pairs_pad = pairs_pad;
  a.n_kb = pairs_pad / 8;
  a.block_stride = block_stride ? block_stride : 1;
  a.bias = bias_sum;
  a.invq = inv_q;
  a.inv_norm = inv_norm;
  a.nq = nq;
  a.keys = keys;
  a.ld = ld;
  a.err = err;
  launch_tc<0>(a, lut, stream);
}

void launch_fastscan_filter_tc(const uint8_t* blocks, uint64_t n, uint32_t pairs_pad, const uint8_t* lut,
                               const float* bias_sum, const float* inv_q, float inv_norm, uint64_t nq,
                               const uint32_t* thr, uint64_t thr_stride, uint32_t* cnt, uint32_t cap,
                               uint32_t* f_keys, uint32_t* f_ids, uint64_t expect_kept, uint32_t* err,
                               cudaStream_t stream) {
  TcArgs a{};
  a.expect_kept = expect_kept;
  a.blocks = blocks;
  a.n = n;
  a.pairs_pad = pairs_pad;
  a.n_kb = pairs_pad / 8;
  a.block_stride = 1;
  a.bias = bias_sum;
  a.invq = inv_q;
  a.inv_norm = inv_norm;
  a.nq = nq;
  a.thr = thr;
  a.thr_stride = thr_stride;
  a.cnt = cnt;
  a.cap = cap;
  a.f_keys = f_keys;
  a.f_ids = f_ids;
  a.err = err;
  launch_tc<0>(a, lut, stream);
}

uint32_t bitmap_tc_kblocks(uint32_t qpv) { return (qpv + 1) / 2; }
uint32_t bitmap_fp4_kblocks(uint32_t qpv) { return (qpv + 3) / 4; }

// The bitmap filter runs on the FP4 tensor cores when its rows fit the FP4
// form and the bitmap family runs on CTA pairs; OVB_BITMAP_FP4=0 keeps int8.
bool bitmap_fp4_usable(uint32_t qpv) {
  const char* e = getenv("OVB_BITMAP_FP4");
  if (e && e[0] == '0') return false;
  return qpv >= 1 && qpv <= tc_fp4_max_words() && tc_form(1) == TcForm::kPair;
}

void launch_bitmap_fp4_query(const uint64_t* qbits, uint64_t nq, uint32_t qpv, uint8_t* out, cudaStream_t stream) {
  if (!nq) return;
  const uint32_t row = bitmap_fp4_kblocks(qpv) * kTcKBytes;
  uint64_t blocks = (nq * row + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  expand_query_nibbles_kernel<<<(unsigned)blocks, 256, 0, stream>>>(qbits, nq, qpv, row, out);
  launched();
}

void launch_bitmap_tc_query(const uint64_t* qbits, uint64_t nq, uint32_t qpv, uint8_t* out, uint32_t* qpop,
                            cudaStream_t stream) {
  if (!nq) return;
  const uint32_t row = bitmap_tc_kblocks(qpv) * kTcKBytes;
  uint64_t blocks = (nq * row + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  expand_query_bits_kernel<<<(unsigned)blocks, 256, 0, stream>>>(qbits, nq, qpv, row, out);
  launched();
  if (qpop) {
    query_popcount_kernel<<<(unsigned)((nq + 255) / 256), 256, 0, stream>>>(qbits, nq, qpv, qpop);
    launched();
  }
}

void launch_bitmap_scan_tc(const uint64_t* words, uint64_t n, uint32_t qpv, uint32_t key_kind, uint32_t n_top,
                           const uint32_t* qpop,
                           const uint8_t* q_bytes, uint64_t nq, uint32_t block_stride, uint32_t* keys, uint64_t ld,
                           uint32_t* err, cudaStream_t stream) {
  TcArgs a{};
  a.blocks = reinterpret_cast<const uint8_t*>(words);
  a.n = n;
  a.qpv = qpv;
  a.n_kb = bitmap_tc_kblocks(qpv);
  a.key_kind = key_kind;
  a.qpop = qpop;
  a.n_top = n_top;
  a.block_stride = block_stride ? block_stride : 1;
  a.nq = nq;
  a.keys = keys;
  a.ld = ld;
  a.err = err;
  launch_tc<1>(a, q_bytes, stream);
}

void launch_bitmap_filter_tc(const uint64_t* words, uint64_t n, uint32_t qpv, uint32_t key_kind, uint32_t n_top,
                             const uint32_t* qpop, const uint8_t* q_bytes, const uint8_t* q_nib, uint64_t nq,
                             const uint32_t* thr, const uint32_t* thr_pos, uint32_t smp_stride, uint64_t thr_stride,
                             uint32_t* cnt, uint32_t cap, uint32_t* f_keys, uint32_t* f_ids, uint32_t* err,
                             cudaStream_t stream) {
  TcArgs a{};
  a.blocks = reinterpret_cast<const uint8_t*>(words);
  a.n = n;
  a.qpv = qpv;
  a.n_kb = bitmap_tc_kblocks(qpv);
  a.key_kind = key_kind;
  a.qpop = qpop;
  a.n_top = n_top;
  a.block_stride = 1;
  a.nq = nq;
  a.thr = thr;
  a.thr_pos = thr_pos;
  a.smp_stride = smp_stride ? smp_stride : 1;
  a.thr_stride = thr_stride;
  a.cnt = cnt;
  a.cap = cap;
  a.f_keys = f_keys;
  a.f_ids = f_ids;
  a.err = err;
  if (q_nib) {
    if (!bitmap_fp4_usable(qpv)) throw std::invalid_argument("bitmap FP4 filter: rows too long for the FP4 form");
    a.n_kb = bitmap_fp4_kblocks(qpv);
    launch_tc_pair<2>(a, q_nib, stream, true);
    return;
  }
  launch_tc<1>(a, q_bytes, stream);
}

void launch_filter_check(const uint32_t* cnt, uint64_t nq, uint32_t need, uint32_t cap, uint32_t* flag,
                         cudaStream_t stream) {
  if (!nq) return;
  filter_check_kernel<<<(unsigned)((nq + 255) / 256), 256, 0, stream>>>(cnt, nq, need, cap, flag);
  launched();
}

}  // namespace ovb
