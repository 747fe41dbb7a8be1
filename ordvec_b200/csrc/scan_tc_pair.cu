// K3-TC / K2-TC on CTA pairs: the FastScan and bitmap tensor-core scans as a
// persistent kernel whose clusters of two CTAs issue tcgen05.mma.cta_group::2.
//
// Why pairs.  One M=256 MMA spans the two SMs of a pair: each SM holds 128 doc
// rows of A and half of the queries' B, and receives its 128 rows x N of the
// accumulator.  Per SM and per MMA that halves the B bytes read from shared
// memory (at M=128 x N=256 one SM's MMA reads 96 of the 128 bytes per clock
// shared memory delivers, and the A builders need the rest), and it halves the
// accumulator to 256 TMEM columns, so each SM holds two: the epilogue of one
// tile overlaps the next tile's mainloop.  Persistence removes the per-CTA
// setup (TMEM allocation, barrier init, the first loads' latency).
//
// Tiles: 256 docs (rank r of the pair: docs [256 d + 128 r, +128)) x nt <= 256
// queries; tile t = cluster + i * clusters, doc tile t / q_tiles, query tile
// t % q_tiles (query tiles inner: a doc tile's codes are reused from L2).
//
// Warp roles (704 threads per CTA):
//   warp 0, lane 0   TMA producer: this CTA's nt/2 B rows of K-block kb ->
//                    stage s (waits its own empty[s]; complete_tx on the
//                    leader's full_b[s], whose expect_tx the leader posts for
//                    both halves)
//   warp 1           TMEM allocation for the pair (both CTAs); on the leader,
//                    lane 0 issues the MMAs: waits the leader's full_a[s] /
//                    full_b[s], 4 MMAs per K-block, commits to both CTAs'
//                    empty[s]; after a tile's last K-block commits to both
//                    CTAs' acc_full[b]; before a tile waits acc_empty[b]
//   warps 2..5       A builders (both CTAs): a thread per doc row, 8 chunks
//                    per K-block, one arrive per warp on the leader's full_a[s]
//   warps 6..21      epilogue (both CTAs): TMEM lane quarter warp % 4, column
//                    quarter (warp - 6) / 4; after reading the accumulator one
//                    arrive per warp on the leader's acc_empty[b]
// Every wait is bounded; a timeout sets bit 0 of *err and the abort flag of
// both CTAs, every role stops issuing work, and both CTAs meet at the final
// cluster barrier before freeing the tensor memory.
//
// Results are the one-CTA kernel's (scan_fastscan_tc.cu), bit for bit: same
// integer accumulators, same key functions and filter rules.
//
// The bitmap filter also runs on the FP4 tensor cores (MODE 2): a set bit is
// the e2m1 value 1.0 (nibble 0b0010), a clear one 0, so an MMA of K=64 packed
// nibbles (kind::mxf4, every ue8m0 block scale 1) sums 64 products of 0/1 into
// an f32 accumulator, exact for overlaps below 2^24, at twice the int8 rate and
// with half the operand bytes.  The scale factors sit in tensor-memory columns
// [224, 256) (A) and [480, 512) (B), all bytes 127, past the two accumulators
// of N <= 224 query columns; non-negative f32 values order like their bit
// patterns, so the epilogue compares the accumulator bits with the f32 bits of
// each query's integer threshold.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "ovb_common.cuh"
#include "ovb_kernels.h"
#include "tc_common.cuh"
#include "tc_scan.cuh"

namespace ovb {

namespace {

using namespace tc;
using namespace tcs;

constexpr int kPBuildWarps = 4;  // warps 2..5: one thread per doc row
constexpr int kPEpiWarps = 16;   // warps 6..21: four per TMEM lane quarter
constexpr int kPThreads = 32 * (2 + kPBuildWarps + kPEpiWarps);
constexpr int kPEpiThreads = kPEpiWarps * 32;
constexpr uint32_t kPMaxN = 256;
constexpr uint32_t kPMaxQ = 1024;        // queries per launch of the pair form (per-query parameters staged once)
constexpr uint32_t kPRowCacheWords = 16;  // bitmap rows of up to 16 words stay in the builders' registers
constexpr uint32_t kPKBytes = 128;
constexpr uint32_t kPTmemCols = 512;
constexpr uint32_t kPF4MaxN = 224;                  // FP4 form: query columns per tile (scale factors above)
// FP4 form: default query columns per tile (balanced: 1,024 queries -> 5 tiles
// of 208; narrower tiles pay the per-tile synchronisation more often)
constexpr uint32_t kPF4TileN = kPF4MaxN;
constexpr uint32_t kSfaCol = 224, kSfbCol = 480;    // FP4 form: scale-factor columns of A and B
constexpr uint32_t kUnitScales = 0x7F7F7F7Fu;       // four ue8m0 bytes of 2^0

// PAIR: CTA pairs, 128 doc rows per CTA, two 256-column accumulators.
// !PAIR: one CTA per SM, 256 doc rows (two M=128 halves) in one 512-column
// accumulator; the next tile's MMAs wait for the epilogue's TMEM reads only.
template <bool PAIR>
struct PT {
  static constexpr uint32_t kRows = PAIR ? 128 : 256;  // doc rows per CTA per tile
  // A: K-block slots (pair form: a bitmap doc tile's whole row when it fits,
  // built once and read by all its query tiles; otherwise a ring); B: a ring
  static constexpr int kASlots = PAIR ? 6 : 3;
  static constexpr int kBStages = PAIR ? 4 : 3;
  static constexpr uint32_t kSegCap = PAIR ? 128 : 192;  // kept entries per epilogue warp per tile
  static constexpr uint32_t kAStage = kRows * kPKBytes;
  static constexpr uint32_t kBStage = (PAIR ? kPMaxN / 2 : kPMaxN) * kPKBytes;
  static constexpr uint32_t kAccBufs = PAIR ? 2 : 1;
  static constexpr uint32_t kRowsPerThread = kRows / (kPBuildWarps * 32);
};

template <bool PAIR>
struct PSmem {
  uint8_t a[PT<PAIR>::kASlots][PT<PAIR>::kAStage];
  uint8_t b[PT<PAIR>::kBStages][PT<PAIR>::kBStage];
  uint2 list[kPEpiWarps][PT<PAIR>::kSegCap];  // (accumulator, q | slot << 8 | row << 16)
  // one-CTA form: per-query parameters of the current tile
  static constexpr uint32_t kTileQ = PAIR ? 1 : kPMaxN;
  float bias[kTileQ];
  float invq[kTileQ];
  uint32_t thr[kTileQ];
  uint32_t amin[kTileQ];
  uint32_t tdoc[kTileQ];
  uint32_t qpop[kTileQ];  // sign bitmaps: query popcounts
  uint32_t cnt[kTileQ];
  uint32_t base[kTileQ];
  // pair form: per-query parameters of the launch, [amin | tdoc or bias | thr | qpop or invq]
  uint32_t qp[PAIR ? 4 * kPMaxQ : 1];
  uint32_t wamin[PAIR ? kPEpiWarps : 1][64];  // pair form: each epilogue warp's 64 column thresholds
  // pair form, bitmap rows of <= kPRowCacheWords words: each builder thread's row
  // of the current doc tile (pitch kPRowCacheWords + 1 words: a warp's 8-byte reads
  // take the minimum two wavefronts)
  uint64_t rowc[PAIR ? 128 : 1][kPRowCacheWords + 1];
  uint64_t full_a[PT<PAIR>::kASlots];
  uint64_t empty_a[PT<PAIR>::kASlots];
  uint64_t full_b[PT<PAIR>::kBStages];
  uint64_t empty_b[PT<PAIR>::kBStages];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint32_t tmem;
  uint32_t abort;
  uint32_t epi_stop;   // epilogue: stop after this tile (written before an epilogue barrier)
  uint32_t seg_full;   // filter: some warp's list segment overflowed in this tile
  uint32_t any_exact;  // filter: some query of this tile needs key compares
};

__device__ __forceinline__ uint32_t cta_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// shared::cluster address of the same object in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t peer_addr(uint32_t local, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}

__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Arrive on a barrier at a cluster address (either CTA of the pair), with the
// instruction's default (release, CTA-scope) semantics: a release at cluster
// scope costs each arriving warp about half a microsecond.
__device__ __forceinline__ void arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}

// Barriers with arrivals from the other CTA are waited like local ones.
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity) { return mbar_wait(bar, parity); }
// Waits of the threads that feed or issue the MMAs: short suspend hints (a
// waiter suspended for long wakes late and the tensor pipe idles meanwhile)
__device__ __forceinline__ bool mbar_wait_issuer(uint64_t* bar, uint32_t parity) { return mbar_wait_spin(bar, parity); }

template <bool PAIR>
__device__ __forceinline__ bool aborted(const PSmem<PAIR>& S) {
  return *reinterpret_cast<const volatile uint32_t*>(&S.abort) != 0;
}

// Sets the abort flag of the CTA (and of its pair) and bit 0 of *err.
template <bool PAIR>
__device__ __forceinline__ void raise_abort(PSmem<PAIR>& S, uint32_t* err) {
  atomicExch(&S.abort, 1u);
  if (PAIR)
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(peer_addr(smem_u32(&S.abort), cta_rank() ^ 1)), "r"(1u)
                 : "memory");
  atomicOr(err, 1u);
}

// TMA tile load of this CTA's B rows; the transaction bytes land on the
// barrier at cluster address `bar` (the leader's).
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
      "%4}], [%2];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void mma_i8_pair(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}


// tcgen05.mma kind::mxf4 across the pair: packed e2m1 A and B, f32 D, one
// ue8m0 scale per 32 K-elements of each row read from tensor memory at sfa /
// sfb; one K=64 step (32 bytes of each row).
__device__ __forceinline__ void mma_mxf4_pair(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                              uint32_t accumulate, uint32_t sfa, uint32_t sfb) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::mxf4.block_scale.block32 [%0], %1, %2, %3, [%5], [%6], p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(sfa), "r"(sfb)
      : "memory");
}

// Stores the word w into 32 consecutive columns from taddr in every lane of the
// calling warp's tensor-memory lane quarter.
__device__ __forceinline__ void tmem_fill32(uint32_t taddr, uint32_t w) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(taddr),
      "r"(w)
      : "memory");
}

// Bits 0..7 of x -> eight nibbles, nibble i = e2m1 1.0 (0b0010) where bit i is
// set and 0 elsewhere (bit i moves to bit 4 i + 1; the shifted copies never
// overlap, so no carries).
__device__ __forceinline__ uint32_t fp4_ones8(uint32_t x) {
  uint32_t v = x & 0xFFu;
  v = (v | (v << 12)) & 0x000F000Fu;
  v = (v | (v << 6)) & 0x03030303u;
  v = (v | (v << 3)) & 0x11111111u;
  return v << 1;
}

// v[j] by a 5-level select tree on the bits of j (no local-memory indexing)
__device__ __forceinline__ uint32_t pick32(const uint32_t (&v)[32], uint32_t j) {
  uint32_t t16[16], t8[8], t4[4], t2[2];
#pragma unroll
  for (uint32_t i = 0; i < 16; i++) t16[i] = (j & 1) ? v[2 * i + 1] : v[2 * i];
#pragma unroll
  for (uint32_t i = 0; i < 8; i++) t8[i] = (j & 2) ? t16[2 * i + 1] : t16[2 * i];
#pragma unroll
  for (uint32_t i = 0; i < 4; i++) t4[i] = (j & 4) ? t8[2 * i + 1] : t8[2 * i];
#pragma unroll
  for (uint32_t i = 0; i < 2; i++) t2[i] = (j & 8) ? t4[2 * i + 1] : t4[2 * i];
  return (j & 16) ? t2[1] : t2[0];
}

// The integer value of an f32 accumulator holding an integer in [0, 2^23)
// (add 2^23: the integer lands in the mantissa bits).
__device__ __forceinline__ uint32_t f4_int(uint32_t bits) {
  return __float_as_uint(__fadd_rn(__uint_as_float(bits), 8388608.0f)) & 0x7FFFFFu;
}

// Arrive-one on the barrier at the same shared-memory offset in both CTAs of
// the pair when every MMA this thread issued so far has completed (a commit
// with a CTA mask: one instruction for both CTAs' barriers).
__device__ __forceinline__ void commit_both(uint32_t local_bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          local_bar),
      "h"((uint16_t)3)
      : "memory");
}

// named barrier 1 over the epilogue warps
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kPEpiThreads) : "memory"); }

struct PairGrid {
  uint32_t n_doc_tiles, q_tiles;
  uint32_t doc_major;  // 1: a cluster takes whole doc tiles, their query tiles back to back
};

// A cluster's walk over its tiles.  doc_major: doc tiles cluster, cluster +
// n_clusters, ..., each with its query tiles 0 .. q_tiles-1 in a row, so a doc
// tile's rows are read once per cluster (the bitmap builders build its A once
// for all its query tiles).  Otherwise tiles cluster + i * n_clusters of the
// doc-major tile order (more clusters busy when there are few doc tiles).  The
// doc-major walk advances without divisions (the issuing threads run it once
// per tile on their critical path); di counts the doc tiles walked before dt.
// The host keeps doc tiles x query tiles below 2^32.
struct TileCursor {
  uint32_t dt, qt, di, tile;
  __device__ __forceinline__ void start(const PairGrid& g, uint32_t cluster) {
    di = 0;
    tile = cluster;
    if (g.doc_major) {
      dt = cluster;
      qt = 0;
    } else {
      dt = tile / g.q_tiles;
      qt = tile - dt * g.q_tiles;
    }
  }
  __device__ __forceinline__ bool valid(const PairGrid& g) const { return dt < g.n_doc_tiles; }
  __device__ __forceinline__ void next(const PairGrid& g, uint32_t n_clusters) {
    if (g.doc_major) {
      if (++qt == g.q_tiles) {
        qt = 0;
        dt += n_clusters;
        di++;
      }
    } else {
      tile += n_clusters;
      dt = tile / g.q_tiles;
      qt = tile - dt * g.q_tiles;
    }
  }
};


template <int MODE, bool PAIR>
__device__ __forceinline__ void pair_body(const CUtensorMap& b_map, const TcArgs& a, const PairGrid g) {
  using T = PT<PAIR>;
  constexpr bool BM = MODE != 0, F4 = MODE == 2;  // bitmap rows; on the FP4 tensor cores
  static_assert(!F4 || PAIR, "the FP4 bitmap form runs on CTA pairs");
  constexpr int kASlots = T::kASlots, kBStages = T::kBStages;
  constexpr uint32_t kPRows = T::kRows, kPSegCap = T::kSegCap, kBufs = T::kAccBufs;
  extern __shared__ uint8_t smem_raw[];
  PSmem<PAIR>& S =
      *reinterpret_cast<PSmem<PAIR>*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const uint32_t rank = PAIR ? cta_rank() : 0u;
  // a "cluster" is a pair of CTAs, or one CTA
  const uint32_t cluster = PAIR ? blockIdx.x >> 1 : blockIdx.x, n_clusters = PAIR ? gridDim.x >> 1 : gridDim.x;
  const uint32_t nt = a.nt, half = nt / 2;
  const uint32_t n_kb = a.n_kb;
  const uint64_t n_blocks = (a.n + 31) / 32;
  const bool dense = a.keys != nullptr;
  // FP4 form: filter only, rows held in the builders' row cache (host-checked;
  // a launch that breaks either does no work and sets bit 0 of *err)
  if (F4 && (dense || a.qpv > kPRowCacheWords || nt > kPF4MaxN)) {
    if (t == 0 && blockIdx.x == 0) atomicOr(a.err, 1u);
    return;
  }
  // A resident per doc tile: built once, read by the doc tile's q_tiles
  // consecutive tiles (whole doc tiles per cluster, rows of <= 12 words)
  const bool resA = PAIR && BM && g.doc_major && n_kb <= (uint32_t)kASlots && a.qpv <= kPRowCacheWords;
  // resident A in two halves when two doc tiles fit: the builders build the
  // next doc tile's rows while the MMAs read the current one's
  const bool resA2 = resA && 2 * n_kb <= (uint32_t)kASlots;

  if (t == 32) {
    for (int s = 0; s < kASlots; s++) {
      mbar_init(&S.full_a[s], (PAIR ? 2 : 1) * kPBuildWarps);  // builder warps of both CTAs
      mbar_init(&S.empty_a[s], 1);                             // the leader's MMA commit
    }
    for (int s = 0; s < kBStages; s++) {
      mbar_init(&S.full_b[s], 1);   // the leader's expect_tx
      mbar_init(&S.empty_b[s], 1);  // the leader's MMA commit
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&S.acc_full[b], 1);
      mbar_init(&S.acc_empty[b], (PAIR ? 2 : 1) * kPEpiWarps);  // epilogue warps of both CTAs
    }
    S.abort = 0;
    S.epi_stop = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    if (PAIR) {
      asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                   "r"(kPTmemCols)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    } else {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                   "r"(kPTmemCols)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  if (PAIR)
    cluster_sync_all();  // both CTAs' barriers initialised, TMEM allocated
  else
    __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S.tmem;
  if constexpr (F4) {
    // unit scale factors in both CTAs before the first MMA: one epilogue warp
    // per tensor-memory lane quarter (warp % 4)
    if (warp >= 2 + kPBuildWarps && warp < 6 + kPBuildWarps) {
      const uint32_t lanes = ((uint32_t)(warp & 3) * 32) << 16;
      tmem_fill32(tmem + lanes + kSfaCol, kUnitScales);
      tmem_fill32(tmem + lanes + kSfbCol, kUnitScales);
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    cluster_sync_all();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }

  if (warp == 0) {
    // ---- TMA producer (both CTAs) ----------------------------------------------
    if (lane == 0) {
      uint64_t it = 0;  // K-blocks issued
      TileCursor tc_;
      for (tc_.start(g, cluster); tc_.valid(g) && !aborted(S); tc_.next(g, n_clusters)) {
        const uint64_t q0 = (uint64_t)tc_.qt * nt;
        for (uint32_t kb = 0; kb < n_kb; kb++, it++) {
          const uint32_t s = (uint32_t)(it % kBStages);
          if (aborted(S)) break;
          if (it >= (uint64_t)kBStages && !mbar_wait_issuer(&S.empty_b[s], (uint32_t)((it / kBStages - 1) & 1))) {
            raise_abort(S, a.err);
            break;
          }
          if (rank == 0) mbar_expect_tx(&S.full_b[s], nt * kPKBytes);  // both halves
          if (PAIR)
            tma_load_2d_pair(S.b[s], &b_map, (int)(kb * kPKBytes), (int)(q0 + rank * half),
                             peer_addr(smem_u32(&S.full_b[s]), 0));
          else
            tma_load_2d(S.b[s], &b_map, (int)(kb * kPKBytes), (int)q0, &S.full_b[s]);
        }
      }
      // the leader waits (bounded) until its last copies, and the peer's, landed
      if (rank == 0)
        for (uint64_t j = it > (uint64_t)kBStages ? it - kBStages : 0; j < it; j++)
          mbar_wait_cluster(&S.full_b[j % kBStages], (uint32_t)((j / kBStages) & 1));
    }
  } else if (warp == 1) {
    // ---- MMA issuer (leader) ------------------------------------------------------
    if (lane == 0 && rank == 0) {
      // i8: D s32, A/B u8, K-major, N = nt; M = 256 across the pair, or two M = 128 halves.
      // FP4: A/B e2m1 (format 1), K-major, ue8m0 scales (bit 23), scale ids 0, K = 64, D f32
      const uint32_t idesc = F4 ? (1u << 7) | (1u << 10) | ((nt >> 3) << 17) | (1u << 23) | (16u << 24)
                                : (2u << 4) | ((nt >> 3) << 17) | ((uint32_t)((PAIR ? 256 : 128) >> 4) << 24);
      uint64_t it = 0, issued = 0;  // B K-blocks issued, last issued B K-block + 1
      uint32_t rb_s = 0, rb_p = 0, ra_s = 0, ra_p = 0;  // B ring / A ring: slot and phase of the next K-block
      uint32_t tcount = 0;
      bool ok = true;
      TileCursor tc_;
      for (tc_.start(g, cluster); tc_.valid(g) && ok; tc_.next(g, n_clusters), tcount++) {
        const uint32_t b = tcount % kBufs;
        // resident A: this doc tile's slots and their phase
        const uint32_t a_base = resA2 ? (tc_.di & 1) * n_kb : 0u;
        const uint32_t pa_res = (resA2 ? tc_.di >> 1 : tc_.di) & 1;
        const bool last_q = tc_.qt + 1 == g.q_tiles;  // resident A: its last reader
        if (tcount >= kBufs && !mbar_wait_issuer(&S.acc_empty[b], (tcount / kBufs - 1) & 1)) ok = false;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + b * 256;
        for (uint32_t kb = 0; kb < n_kb && ok; kb++, it++) {
          const uint32_t sb = rb_s, pb = rb_p;
          const uint32_t sa = resA ? a_base + kb : ra_s;
          const uint32_t pa = resA ? pa_res : ra_p;
          // resident A: after the doc tile's first query tile its slots are known
          // full (nothing refills them before its last query tile frees them)
          const bool need_a = !resA || tc_.qt == 0;
          if ((kb == 0 && aborted(S)) || !mbar_wait_issuer(&S.full_b[sb], pb) ||
              (need_a && !mbar_wait_issuer(&S.full_a[sa], pa))) {
            ok = false;
            break;
          }
          // (operands arrive by TMA, or by builder stores behind a proxy fence and
          // the barrier: no tcgen05 fence is needed before reading them)
          if (!PAIR) asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = smem_u32(S.a[sa]), b0 = smem_u32(S.b[sb]);
          const bool free_a = !resA || last_q;
          if (PAIR) {
            // a 32-byte K step adds 2 to the descriptor's start-address field (16-byte units)
            const uint64_t ad = sw128_desc(a0), bd = sw128_desc(b0);
            if constexpr (F4) {
#pragma unroll
              for (uint32_t j = 0; j < 4; j++)
                mma_mxf4_pair(d, ad + 2 * j, bd + 2 * j, idesc, (kb | j) != 0, tmem + kSfaCol, tmem + kSfbCol);
            } else {
#pragma unroll
              for (uint32_t j = 0; j < 4; j++) mma_i8_pair(d, ad + 2 * j, bd + 2 * j, idesc, (kb | j) != 0);
            }
            commit_both(smem_u32(&S.empty_b[sb]));
            if (free_a) commit_both(smem_u32(&S.empty_a[sa]));
          } else {
#pragma unroll
            for (uint32_t j = 0; j < 4; j++) {
              const uint64_t bd = sw128_desc(b0 + 32 * j);
              mma_i8(d, sw128_desc(a0 + 32 * j), bd, idesc, (kb | j) != 0);
              mma_i8(d + 256, sw128_desc(a0 + kPRows / 2 * kPKBytes + 32 * j), bd, idesc, (kb | j) != 0);
            }
            mma_commit(&S.empty_b[sb]);
            mma_commit(&S.empty_a[sa]);
          }
          if (!resA && ++ra_s == (uint32_t)kASlots) {
            ra_s = 0;
            ra_p ^= 1;
          }
          if (++rb_s == (uint32_t)kBStages) {
            rb_s = 0;
            rb_p ^= 1;
          }
          issued = it + 1;
        }
        if (!ok) break;
        if (PAIR) {
          commit_both(smem_u32(&S.acc_full[b]));
        } else {
          mma_commit(&S.acc_full[b]);
        }
      }
      if (!ok) {
        if (!aborted(S)) raise_abort(S, a.err);
        // no MMA in flight when the pair frees its tensor memory
        if (issued > 0)
          mbar_wait(&S.empty_b[(issued - 1) % kBStages], (uint32_t)(((issued - 1) / kBStages) & 1));
      }
    }
  } else if (warp < 2 + kPBuildWarps) {
    // ---- A builders: thread r builds doc rows r + 128 i (i < kRowsPerThread), chunks 0..7
    constexpr uint32_t R = T::kRowsPerThread;
    const uint32_t r = (uint32_t)t - 64;  // 0..127
    // leader's full_a[0] (a cluster address; the CTA's own barrier when alone)
    const uint32_t full_a0 = PAIR ? peer_addr(smem_u32(&S.full_a[0]), 0) : 0u;
    uint64_t it = 0;
    bool ok = true;
    // wait for A ring slot s to be free, or stop (warp-uniform)
    auto acquire = [&](uint32_t s) -> bool {
      bool w = true;
      if (it >= (uint64_t)kASlots) {
        if (lane == 0) w = !aborted(S) && mbar_wait_issuer(&S.empty_a[s], (uint32_t)((it / kASlots - 1) & 1));
        w = __shfl_sync(0xFFFFFFFFu, w, 0);
        if (!w && lane == 0 && !aborted(S)) raise_abort(S, a.err);
        __syncwarp();
      }
      return w;
    };
    auto publish = [&](uint32_t s) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        if (PAIR)
          arrive_remote(full_a0 + 8 * s);
        else
          mbar_arrive(&S.full_a[s]);
      }
    };
    uint64_t cached_dt = ~0ull;  // pair form, bitmap rows <= 16 words: doc tile of S.rowc
    TileCursor tc_;
    for (tc_.start(g, cluster); tc_.valid(g) && ok; tc_.next(g, n_clusters)) {
      const uint64_t dt = tc_.dt;
      const uint32_t qt_ = tc_.qt;
      uint64_t pb[R], doc[R];
      uint32_t a_row[R];  // row offset in a stage: 8-row atoms of 1024 bytes, 128 bytes a row
#pragma unroll
      for (uint32_t i = 0; i < R; i++) {
        const uint32_t row = r + 128 * i;
        pb[i] = (dt * 8 + rank * (kPRows / 32) + (row >> 5)) * a.block_stride;
        doc[i] = pb[i] * 32 + (row & 31);
        a_row[i] = (row >> 3) * 1024 + (row & 7) * 128;
      }
      if constexpr (BM && PAIR) {
        if (a.qpv <= kPRowCacheWords) {
          // the row's words stay in registers while the doc tile's query tiles pass
          if (dt != cached_dt) {
            const bool row_ok = pb[0] < n_blocks && doc[0] < a.n;
            const uint64_t* wp = reinterpret_cast<const uint64_t*>(a.blocks) + (row_ok ? doc[0] : 0) * (uint64_t)a.qpv;
            // global -> shared without registers; words past the row (or of an
            // invalid row) are zero-filled (source size 0)
#pragma unroll
            for (uint32_t j = 0; j < kPRowCacheWords; j++) {
              const uint32_t src_bytes = (row_ok && j < a.qpv) ? 8u : 0u;
              asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(&S.rowc[r][j])),
                           "l"(wp + (src_bytes ? j : 0)), "r"(src_bytes)
                           : "memory");
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            cached_dt = dt;
            // warm L2 with the row of this cluster's next doc tile
            const uint64_t nd = dt + n_clusters;
            if (nd < g.n_doc_tiles) {
              const uint64_t npb = (nd * 8 + rank * (kPRows / 32) + (r >> 5)) * a.block_stride;
              const uint64_t ndoc = npb * 32 + (r & 31);
              if (npb < n_blocks && ndoc < a.n)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const uint64_t*>(a.blocks) +
                                                             ndoc * (uint64_t)a.qpv));
            }
          }
          if (resA && qt_ != 0) continue;  // the doc tile's A is resident: built at its first query tile
          // resident A: earlier uses of this doc tile's slots (doc tiles this
          // cluster started before, or of the same parity with two halves)
          const uint64_t dc = resA2 ? tc_.di >> 1 : tc_.di;
          const uint32_t s_base = resA2 ? (tc_.di & 1) * n_kb : 0u;
          const uint32_t base0 = a_row[0], rr = r & 7;
          constexpr uint32_t kWordsPerKb = F4 ? 4 : 2;  // 128 bytes: 256 nibbles or 128 bytes of 0/1
#pragma unroll
          for (uint32_t kb = 0; kb < kPRowCacheWords / kWordsPerKb; kb++) {
            if (kb >= n_kb) break;
            uint32_t s;
            if (resA) {
              s = s_base + kb;
              if (dc > 0) {  // the slot's previous doc tile has been read by its last query tile
                // (with two halves the builders run a doc tile ahead: they sleep
                // rather than poll, leaving the issue slots to the epilogue and MMA warps)
                bool w = true;
                if (lane == 0)
                  w = !aborted(S) && (resA2 ? mbar_wait(&S.empty_a[s], (uint32_t)((dc - 1) & 1))
                                            : mbar_wait_issuer(&S.empty_a[s], (uint32_t)((dc - 1) & 1)));
                w = __shfl_sync(0xFFFFFFFFu, w, 0);
                if (!w && lane == 0 && !aborted(S)) raise_abort(S, a.err);
                __syncwarp();
                if (!w) {
                  ok = false;
                  break;
                }
              }
            } else {
              s = (uint32_t)(it % kASlots);
              if (!acquire(s)) {
                ok = false;
                break;
              }
            }
            const uint32_t base = smem_u32(S.a[s]) + base0;
            if constexpr (F4) {
#pragma unroll
              for (uint32_t c = 0; c < 8; c++) {  // 32 coordinates (half a word) per 16-byte chunk
                const uint32_t h = (uint32_t)(S.rowc[r][4 * kb + (c >> 1)] >> (32 * (c & 1)));
                st_shared_v4(base + ((c ^ rr) << 4), fp4_ones8(h), fp4_ones8(h >> 8), fp4_ones8(h >> 16),
                             fp4_ones8(h >> 24));
              }
            } else {
              const uint64_t w0 = S.rowc[r][2 * kb], w1 = S.rowc[r][2 * kb + 1];
#pragma unroll
              for (uint32_t c = 0; c < 8; c++) {  // 16 coordinates per 16-byte chunk
                const uint32_t h = (uint32_t)((c < 4 ? w0 : w1) >> (16 * (c & 3)));
                uint32_t o[4];
#pragma unroll
                for (uint32_t q = 0; q < 4; q++) o[q] = (((h >> (4 * q)) & 15u) * 0x00204081u) & 0x01010101u;
                st_shared_v4(base + ((c ^ rr) << 4), o[0], o[1], o[2], o[3]);
              }
            }
            publish(s);
            it++;
          }
          continue;
        }
      }
      if constexpr (MODE == 1) {
        const uint64_t* words[R];
        bool row_ok[R];
        uint64_t w[R][4];  // K-block kb = words 2 kb, 2 kb + 1; two K-blocks of words in flight
#pragma unroll
        for (uint32_t i = 0; i < R; i++) {
          row_ok[i] = pb[i] < n_blocks && doc[i] < a.n;
          words[i] = reinterpret_cast<const uint64_t*>(a.blocks) + (row_ok[i] ? doc[i] : 0) * (uint64_t)a.qpv;
#pragma unroll
          for (uint32_t j = 0; j < 4; j++) w[i][j] = (row_ok[i] && j < a.qpv) ? __ldg(words[i] + j) : 0ull;
        }
        for (uint32_t kb = 0; kb < n_kb; kb++, it++) {
          uint64_t lo[R], hi[R];
#pragma unroll
          for (uint32_t i = 0; i < R; i++) {
            lo[i] = w[i][0];
            hi[i] = w[i][1];
            w[i][0] = w[i][2];
            w[i][1] = w[i][3];
            const uint32_t wi = 2 * kb + 4;
            w[i][2] = (row_ok[i] && wi < a.qpv) ? __ldg(words[i] + wi) : 0ull;
            w[i][3] = (row_ok[i] && wi + 1 < a.qpv) ? __ldg(words[i] + wi + 1) : 0ull;
          }
          const uint32_t s = (uint32_t)(it % kASlots);
          if (!acquire(s)) {
            ok = false;
            break;
          }
#pragma unroll
          for (uint32_t i = 0; i < R; i++) {
            const uint32_t base = smem_u32(S.a[s]) + a_row[i], rr = (r + 128 * i) & 7;
#pragma unroll
            for (uint32_t c = 0; c < 8; c++) {  // 16 coordinates per 16-byte chunk
              const uint32_t h = (uint32_t)((c < 4 ? lo[i] : hi[i]) >> (16 * (c & 3)));
              uint32_t o[4];
#pragma unroll
              for (uint32_t q = 0; q < 4; q++)  // 4 bits -> 4 bytes (the shifted copies never overlap)
                o[q] = (((h >> (4 * q)) & 15u) * 0x00204081u) & 0x01010101u;
              st_shared_v4(base + ((c ^ rr) << 4), o[0], o[1], o[2], o[3]);
            }
          }
          publish(s);
        }
      } else if constexpr (MODE == 0) {
        const uint8_t* row_codes[R];
        bool row_valid[R];
        uint4 next[R];
#pragma unroll
        for (uint32_t i = 0; i < R; i++) {
          row_valid[i] = pb[i] < n_blocks;
          row_codes[i] = a.blocks + pb[i] * (uint64_t)a.pairs_pad * 16 + (uint64_t)((r + 128 * i) & 31) * 16;
          next[i] = row_valid[i] ? load_codes(row_codes[i]) : make_uint4(0, 0, 0, 0);
        }
        const uint32_t n_groups = n_kb / 4;  // one 16-byte code load covers 4 K-blocks
        for (uint32_t gi = 0; gi < n_groups && ok; gi++) {
          uint4 chunk[R];
#pragma unroll
          for (uint32_t i = 0; i < R; i++) {
            chunk[i] = next[i];
            if (row_valid[i] && gi + 1 < n_groups) next[i] = load_codes(row_codes[i] + (uint64_t)(gi + 1) * 512);
          }
#pragma unroll
          for (uint32_t j = 0; j < 4; j++) {
            const uint32_t s = (uint32_t)(it % kASlots);
            if (!acquire(s)) {
              ok = false;
              break;
            }
#pragma unroll
            for (uint32_t i = 0; i < R; i++) {
              const uint32_t wv = j == 0 ? chunk[i].x : j == 1 ? chunk[i].y : j == 2 ? chunk[i].z : chunk[i].w;
              const uint32_t base = smem_u32(S.a[s]) + a_row[i], rr = (r + 128 * i) & 7;
#pragma unroll
              for (uint32_t c = 0; c < 8; c++) {
                const uint32_t sh = c == 0 ? (wv << 3) & 0x78u : (wv >> (4 * c - 3)) & 0x78u;  // 8 * nibble c
                st_shared_v4(base + ((c ^ rr) << 4), shl1(sh), shl1(sh - 32), shl1(sh - 64), shl1(sh - 96));
              }
            }
            publish(s);
            it++;
          }
        }
      }
    }
  } else if constexpr (PAIR) {
    // ---- epilogue of the pair form: every warp works alone -----------------------
    // Per-query parameters are staged once per launch (nq <= kPMaxQ); per tile a
    // warp derives the thresholds of its 64 columns, reads its two 32-column
    // accumulator chunks (both loads in flight), keeps the passing entries in
    // its list, releases the accumulator and reserves each entry's slot with a
    // global atomic: no block barrier per tile.
    const uint32_t e = (uint32_t)warp - 2 - kPBuildWarps;  // 0..15
    const uint32_t et = (uint32_t)t - 32 * (2 + kPBuildWarps);
    const uint32_t lq = (uint32_t)warp & 3;  // TMEM lane quarter (hardware rule: warp % 4)
    // this warp's accumulator columns: 64, or 32 for FP4 tiles of <= 128 queries
    // (one 32-column load a warp: the accumulator is released after one read)
    const uint32_t wcols = (F4 && nt <= 128) ? 32u : 64u;
    const uint32_t col0 = (e >> 2) * wcols;
    const uint32_t row = lq * 32 + lane;
    const uint32_t acc_empty0 = peer_addr(smem_u32(&S.acc_empty[0]), 0);
    // S.qp: [amin | tdoc (bitmap) or bias (FastScan) | thr | qpop (bitmap) or invq (FastScan)] x kPMaxQ
#define P_am(i) S.qp[(i)]
#define P_td(i) S.qp[kPMaxQ + (i)]
#define P_thr(i) S.qp[2 * kPMaxQ + (i)]
#define P_pop(i) S.qp[3 * kPMaxQ + (i)]
#define P_bias(i) (*reinterpret_cast<float*>(&S.qp[kPMaxQ + (i)]))
#define P_invq(i) (*reinterpret_cast<float*>(&S.qp[3 * kPMaxQ + (i)]))
    for (uint32_t i = et; i < a.nq && i < kPMaxQ; i += kPEpiThreads) {
      const float bias = MODE == 0 ? a.bias[i] : 0.0f, invq = MODE == 0 ? a.invq[i] : 0.0f;
      const uint32_t qpop = (BM && a.key_kind == 2) ? a.qpop[i] : 0u;
      uint32_t thr = dense ? 0u : a.thr[i * a.thr_stride], am = 0, td = 0;
      if (!dense) {
        if (MODE == 0) {
          am = filter_amin(bias, invq, a.inv_norm, thr, 255u * a.pairs_pad);
        } else {
          am = bm_amin_q(a, qpop, thr);
          if (a.thr_pos) {  // (key, doc) <= (thr, tdoc): the tie level depends on the tile's doc range
            const uint32_t p = a.thr_pos[i * a.thr_stride];
            td = (uint32_t)(((uint64_t)(p >> 5) * a.smp_stride) * 32 + (p & 31));
            thr = am;
          }
        }
      }
      P_am(i) = am;
      P_thr(i) = thr;
      if (MODE == 0) {
        P_bias(i) = bias;
        P_invq(i) = invq;
      } else {
        P_td(i) = td;
        P_pop(i) = qpop;
      }
    }
    epi_sync();
    uint2* list = S.list[e];
    uint32_t lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    const uint32_t nch = col0 >= nt ? 0u : (col0 + 32 >= nt || wcols == 32 ? 1u : 2u);  // 32-column chunks (warp-uniform)
    // A tile's kept entries -> the candidate rows: a slot per entry by a global
    // atomic on its query's count; a list that overflowed fails every query of
    // the warp's columns (bit 31 > cap).
    auto flush = [&](uint32_t wcount, uint64_t q0, uint64_t dt, uint32_t nqt) {
      __syncwarp();
      if (wcount > kPSegCap) {
        for (uint32_t j = lane; j < wcols; j += 32)
          if (col0 + j < nqt) atomicOr(&a.cnt[q0 + col0 + j], 0x80000000u);
      }
      const uint32_t tot = wcount < kPSegCap ? wcount : kPSegCap;
      for (uint32_t j = lane; j < tot; j += 32) {
        const uint2 en = list[j];
        const uint32_t q = en.y & 0xFFFFu, rw_ = en.y >> 16;
        const uint32_t pos = atomicAdd(&a.cnt[q0 + q], 1u);
        if (pos < a.cap) {
          a.f_keys[(q0 + q) * a.cap + pos] = MODE == 0
              ? desc_key(tc_score(en.x, P_bias(q0 + q), P_invq(q0 + q), a.inv_norm))
              : bm_key_q(a, P_pop(q0 + q), en.x);
          const uint64_t rpb = (dt * 8 + rank * (kPRows / 32) + (rw_ >> 5)) * a.block_stride;
          a.f_ids[(q0 + q) * a.cap + pos] = (uint32_t)(rpb * 32 + (rw_ & 31));
        }
      }
      __syncwarp();  // the list is reused by the next tile
    };
    if constexpr (F4) {
      // FP4 form: the f32 sums of constant-weight and multi-bucket keys are
      // compared as bits with the f32 bits of each column's integer threshold
      // (non-negative floats order like their bit patterns); sign bitmaps take
      // the integer sums.  Both 32-column chunks are read back to back (one
      // tensor-memory latency) and the buffer released before any compare; the
      // slots of a tile's kept entries are reserved by atomics whose results are
      // first used during the next tile.
      uint32_t* wam = S.wamin[e];
      const bool fbits = a.key_kind != 2;
      // this lane's entry of the previous tile, its slot reserved
      bool pend = false;
      uint32_t p_pos = 0, p_key = 0, p_id = 0;
      uint64_t p_q = 0;
      auto finish = [&]() {
        if (pend && p_pos < a.cap) {
          a.f_keys[p_q * a.cap + p_pos] = p_key;
          a.f_ids[p_q * a.cap + p_pos] = p_id;
        }
        pend = false;
      };
      uint32_t tcount = 0;
      TileCursor tc_;
      for (tc_.start(g, cluster); tc_.valid(g); tc_.next(g, n_clusters), tcount++) {
        const uint64_t dt = tc_.dt;
        const uint64_t q0 = (uint64_t)tc_.qt * nt;
        const uint32_t nqt = (uint32_t)((a.nq - q0) < nt ? (a.nq - q0) : nt);
        const uint32_t b = tcount % kBufs;
        const uint64_t first = dt * 256 + rank * kPRows;
        // thresholds of this warp's columns for this tile
#pragma unroll
        for (uint32_t h2 = 0; h2 < 2; h2++) {
          const uint32_t c = col0 + 32 * h2 + lane;
          uint32_t am = kNeverPasses;
          if (c < nqt) {
            am = P_am(q0 + c);
            if (a.thr_pos) {
              const uint32_t td = P_td(q0 + c);
              am = td >= first + kPRows - 1 ? am : td < first ? am + 1 : kExactCompare;
            }
            if (fbits && am < kNeverPasses) am = __float_as_uint((float)am);  // exact: am <= 2^24
          }
          wam[32 * h2 + lane] = am;
        }
        const bool any_exact = __any_sync(0xFFFFFFFFu, wam[lane] == kExactCompare || wam[32 + lane] == kExactCompare);
        __syncwarp();
        bool ready = false;
        if (lane == 0) ready = !aborted(S) && mbar_wait_cluster(&S.acc_full[b], (tcount / kBufs) & 1);
        ready = __shfl_sync(0xFFFFFFFFu, ready, 0);
        if (!ready) {
          if (lane == 0 && !aborted(S)) raise_abort(S, a.err);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint64_t doc = first + row;  // filter: block stride 1
        const bool valid = doc < a.n;
        const uint32_t taddr = tmem + ((lq * 32) << 16) + b * 256 + col0;
        const uint32_t dpop = fbits ? 0u : row_popcount(a, doc, valid);
        uint32_t wcount = 0;
        if (nch == 0) {  // nothing to read: release the accumulator at once
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) arrive_remote(acc_empty0 + 8 * b);
        }
        for (uint32_t c = 0; c < nch; c++) {
          const uint32_t cb = col0 + 32 * c;
          uint32_t v[32];
          __syncwarp();
          tmem_ld32(taddr + 32 * c, v);
          if (c + 1 == nch) {  // the last chunk is in registers: release the accumulator to the MMAs
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) arrive_remote(acc_empty0 + 8 * b);
          }
          if (c == 0) finish();  // the previous tile's slots have long been reserved
          if (!fbits) {
#pragma unroll
            for (uint32_t j = 0; j < 32; j++) v[j] = ham_y(f4_int(v[j]), dpop);
          }
          uint32_t hm = 0;  // the columns (queries) this lane's doc passes
          if (!any_exact) {
#pragma unroll
            for (uint32_t j = 0; j < 32; j += 4) {
              const uint4 am = *reinterpret_cast<const uint4*>(&wam[32 * c + j]);
              hm |= ((uint32_t)(v[j] >= am.x) << j) | ((uint32_t)(v[j + 1] >= am.y) << (j + 1)) |
                    ((uint32_t)(v[j + 2] >= am.z) << (j + 2)) | ((uint32_t)(v[j + 3] >= am.w) << (j + 3));
            }
          } else {
#pragma unroll
            for (uint32_t j = 0; j < 32; j++) {
              const uint32_t q = (uint32_t)q0 + cb + j;
              const uint32_t am = wam[32 * c + j];
              const uint32_t tq = fbits ? __float_as_uint((float)P_thr(q)) : P_thr(q);
              const bool pass = am != kExactCompare ? v[j] >= am : v[j] > tq || (v[j] == tq && doc <= P_td(q));
              hm |= (uint32_t)pass << j;
            }
          }
          // columns past the tile's queries (never written by the MMAs) keep nothing
          if (!valid) hm = 0;
          const uint32_t ncols = nqt > cb ? nqt - cb : 0u;
          hm &= ncols >= 32 ? 0xFFFFFFFFu : (1u << ncols) - 1u;
          while (__any_sync(0xFFFFFFFFu, hm != 0)) {
            const bool has = hm != 0;
            const uint32_t j = has ? (uint32_t)(__ffs(hm) - 1) : 0u;
            const uint32_t bal = __ballot_sync(0xFFFFFFFFu, has);
            const uint32_t pos = wcount + __popc(bal & lt);
            if (has && pos < kPSegCap) {
              const uint32_t x = pick32(v, j);
              list[pos] = make_uint2(fbits ? (uint32_t)__uint_as_float(x) : x, (cb + j) | (row << 16));
            }
            wcount += __popc(bal);
            hm &= hm - 1;
          }
        }
        if (nch == 0) finish();
        __syncwarp();
        if (wcount > 32) {
          flush(wcount, q0, dt, nqt);  // more than one entry per lane (or lost ones): reserve and write now
        } else if (lane < wcount) {
          // reserve this lane's slot now, write the entry during the next tile
          const uint2 en = list[lane];
          const uint32_t q = en.y & 0xFFFFu, rw_ = en.y >> 16;
          p_q = q0 + q;
          p_pos = atomicAdd(&a.cnt[p_q], 1u);
          p_key = bm_key_q(a, P_pop(p_q), en.x);
          p_id = (uint32_t)(first + rw_);
          pend = true;
        }
        __syncwarp();  // the list is reused by the next tile
      }
      finish();
    } else {
      uint32_t* wam = S.wamin[e];
      uint32_t tcount = 0;
      TileCursor tc_;
      for (tc_.start(g, cluster); tc_.valid(g); tc_.next(g, n_clusters), tcount++) {
        const uint64_t dt = tc_.dt;
        const uint32_t qt_ = tc_.qt;
        const uint64_t q0 = (uint64_t)qt_ * nt;
        const uint32_t nqt = (uint32_t)((a.nq - q0) < nt ? (a.nq - q0) : nt);
        const uint32_t b = tcount % kBufs;
        const uint64_t first = dt * 256 + rank * kPRows;
        // thresholds of this warp's columns for this tile
#pragma unroll
        for (uint32_t h2 = 0; h2 < 2; h2++) {
          const uint32_t c = col0 + 32 * h2 + lane;
          uint32_t am = kNeverPasses;
          if (c < nqt) {
            am = P_am(q0 + c);
            if (BM && a.thr_pos && !dense) {
              const uint32_t td = P_td(q0 + c);
              am = td >= first + kPRows - 1 ? am : td < first ? am + 1 : kExactCompare;
            }
          }
          wam[32 * h2 + lane] = am;
        }
        const bool any_exact = __any_sync(0xFFFFFFFFu, wam[lane] == kExactCompare || wam[32 + lane] == kExactCompare);
        __syncwarp();
        bool ready = false;
        if (lane == 0) ready = !aborted(S) && mbar_wait_cluster(&S.acc_full[b], (tcount / kBufs) & 1);
        ready = __shfl_sync(0xFFFFFFFFu, ready, 0);
        if (!ready) {
          if (lane == 0 && !aborted(S)) raise_abort(S, a.err);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint64_t pb = (dt * 8 + rank * (kPRows / 32) + (row >> 5)) * a.block_stride;
        const uint64_t doc = pb * 32 + lane;
        const uint64_t u = dt * 256 + rank * kPRows + row;
        const bool valid = pb < n_blocks && doc < a.n;
        const uint32_t dpop = (BM && a.key_kind == 2) ? row_popcount(a, doc, valid) : 0u;
        const uint32_t taddr = tmem + ((lq * 32) << 16) + b * 256 + col0;
        uint32_t wcount = 0;
        if (nch == 0) {  // nothing to read: release the accumulator at once
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) arrive_remote(acc_empty0 + 8 * b);
        }
        for (uint32_t c = 0; c < nch; c++) {
          const uint32_t cb = col0 + 32 * c;
          uint32_t v[32];
          __syncwarp();
          tmem_ld32(taddr + 32 * c, v);
          if (c + 1 == nch) {  // the last chunk is in registers: release the accumulator to the MMA
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) arrive_remote(acc_empty0 + 8 * b);
          }
          if (BM && a.key_kind == 2) {
#pragma unroll
            for (uint32_t j = 0; j < 32; j++) v[j] = ham_y(v[j], dpop);
          }
          if (dense) {
#pragma unroll
            for (uint32_t j = 0; j < 32; j++) {
              const uint32_t q = cb + j;
              if (valid && q < nqt)
                a.keys[(q0 + q) * a.ld + u] = MODE == 0
                    ? desc_key(tc_score(v[j], P_bias(q0 + q), P_invq(q0 + q), a.inv_norm))
                    : bm_key_q(a, P_pop(q0 + q), v[j]);
            }
            continue;
          }
          uint32_t hm = 0;  // the columns (queries) this lane's doc passes
          if (!any_exact) {
#pragma unroll
            for (uint32_t j = 0; j < 32; j += 4) {
              const uint4 am = *reinterpret_cast<const uint4*>(&wam[32 * c + j]);
              hm |= ((uint32_t)(v[j] >= am.x) << j) | ((uint32_t)(v[j + 1] >= am.y) << (j + 1)) |
                    ((uint32_t)(v[j + 2] >= am.z) << (j + 2)) | ((uint32_t)(v[j + 3] >= am.w) << (j + 3));
            }
          } else {
#pragma unroll
            for (uint32_t j = 0; j < 32; j++) {
              const uint32_t q = q0 + cb + j;
              const uint32_t am = wam[32 * c + j];
              bool pass;
              if (am != kExactCompare)
                pass = v[j] >= am;
              else if (MODE == 0)
                pass = desc_key(tc_score(v[j], P_bias(q), P_invq(q), a.inv_norm)) <= P_thr(q);
              else
                pass = v[j] > P_thr(q) || (v[j] == P_thr(q) && doc <= P_td(q));
              hm |= (uint32_t)pass << j;
            }
          }
          // columns past the tile's queries (never written by the MMAs) keep nothing
          if (!valid) hm = 0;
          const uint32_t ncols = nqt > cb ? nqt - cb : 0u;
          hm &= ncols >= 32 ? 0xFFFFFFFFu : (1u << ncols) - 1u;
          while (__any_sync(0xFFFFFFFFu, hm != 0)) {
            const bool has = hm != 0;
            const uint32_t j = has ? (uint32_t)(__ffs(hm) - 1) : 0u;
            const uint32_t bal = __ballot_sync(0xFFFFFFFFu, has);
            const uint32_t pos = wcount + __popc(bal & lt);
            if (has && pos < kPSegCap) list[pos] = make_uint2(pick32(v, j), (cb + j) | (row << 16));
            wcount += __popc(bal);
            hm &= hm - 1;
          }
        }
        if (!dense) flush(wcount, q0, dt, nqt);
      }
    }
#undef P_am
#undef P_td
#undef P_thr
#undef P_pop
#undef P_bias
#undef P_invq
  } else {
    // ---- epilogue (both CTAs) -------------------------------------------------------
    const uint32_t e = (uint32_t)warp - 2 - kPBuildWarps;  // 0..15
    const uint32_t et = (uint32_t)t - 32 * (2 + kPBuildWarps);
    // TMEM lane quarter (hardware rule: warp % 4); PAIR: column quarter e / 4 of
    // the CTA's 128 rows; !PAIR: accumulator half (rows 0..127 | 128..255) and
    // column half
    const uint32_t lq = (uint32_t)warp & 3;
    const uint32_t h = PAIR ? 0u : (e >> 2) & 1;
    const uint32_t col0 = PAIR ? (e >> 2) * 64 : (e >> 3) * 128;
    constexpr uint32_t kChunks = PAIR ? 2 : 4;  // 32-column chunks per warp
    const uint32_t row = h * 128 + lq * 32 + lane;
    const uint32_t acc_empty0 = PAIR ? peer_addr(smem_u32(&S.acc_empty[0]), 0) : 0u;
    uint2* list = S.list[e];
    uint32_t lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    uint32_t tcount = 0;
    TileCursor tc_;
    for (tc_.start(g, cluster); tc_.valid(g); tc_.next(g, n_clusters), tcount++) {
      const uint64_t dt = tc_.dt;
      const uint32_t qt_ = tc_.qt;
      const uint64_t q0 = (uint64_t)qt_ * nt;
      const uint32_t nqt = (uint32_t)((a.nq - q0) < nt ? (a.nq - q0) : nt);
      const uint32_t b = tcount % kBufs;
      // per-query parameters of this tile (the previous tile's slot passes are done)
      epi_sync();
      if (et == 0) {
        S.seg_full = 0;
        S.any_exact = 0;
      }
      {
        const uint32_t i = et;  // one query per epilogue thread (nt <= 256)
        const bool v = i < nqt;
        if (i < kPMaxN) {
          S.bias[i] = (MODE == 0 && v) ? a.bias[q0 + i] : 0.0f;
          S.invq[i] = (MODE == 0 && v) ? a.invq[q0 + i] : 0.0f;
          S.thr[i] = (v && !dense) ? a.thr[(q0 + i) * a.thr_stride] : 0u;
          S.qpop[i] = (MODE == 1 && v && a.key_kind == 2) ? a.qpop[q0 + i] : 0u;
          S.cnt[i] = 0;
          uint32_t am;
          if (!v)
            am = kNeverPasses;
          else if (dense)
            am = 0;
          else if (MODE == 0)
            am = filter_amin(S.bias[i], S.invq[i], a.inv_norm, S.thr[i], 255u * a.pairs_pad);
          else {
            am = bm_amin_q(a, S.qpop[i], S.thr[i]);
            if (a.thr_pos) {  // (key, doc) <= (thr, tdoc): tie level by this CTA's doc range
              const uint32_t p = a.thr_pos[(q0 + i) * a.thr_stride];
              const uint64_t td = ((uint64_t)(p >> 5) * a.smp_stride) * 32 + (p & 31);
              const uint64_t first = dt * 256 + rank * kPRows;
              S.tdoc[i] = (uint32_t)td;
              S.thr[i] = am;
              am = td >= first + kPRows - 1 ? am : td < first ? am + 1 : kExactCompare;
            }
          }
          S.amin[i] = am;
        }
      }
      epi_sync();
      for (uint32_t i = et; i < kPMaxN; i += kPEpiThreads)
        if (S.amin[i] == kExactCompare) atomicOr(&S.any_exact, 1u);
      // wait for the accumulator; one verdict for all epilogue warps
      bool ready = false;
      if (lane == 0) ready = !aborted(S) && mbar_wait_cluster(&S.acc_full[b], (tcount / kBufs) & 1);
      ready = __shfl_sync(0xFFFFFFFFu, ready, 0);
      if (!ready && lane == 0) {
        if (!aborted(S)) raise_abort(S, a.err);
        atomicExch(&S.epi_stop, 1u);
      }
      epi_sync();
      if (*reinterpret_cast<volatile uint32_t*>(&S.epi_stop)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint64_t pb = (dt * 8 + rank * (kPRows / 32) + (row >> 5)) * a.block_stride;
      const uint64_t doc = pb * 32 + lane;
      const uint64_t u = dt * 256 + rank * kPRows + row;
      const bool valid = pb < n_blocks && doc < a.n;
      const uint32_t dpop = (MODE == 1 && a.key_kind == 2) ? row_popcount(a, doc, valid) : 0u;
      const uint32_t taddr = tmem + ((lq * 32) << 16) + (b + h) * 256;
      const bool any_exact = S.any_exact != 0;
      uint32_t wcount = 0;
      for (uint32_t c = 0; c < kChunks; c++) {
        const uint32_t cb = col0 + c * 32;
        if (cb >= nt) break;  // warp-uniform
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
        uint32_t hm = 0;  // queries this lane's doc passes
        if (!any_exact) {
#pragma unroll
          for (uint32_t j = 0; j < 32; j += 4) {
            const uint4 am = *reinterpret_cast<const uint4*>(&S.amin[cb + j]);
            hm |= ((uint32_t)(v[j] >= am.x) << j) | ((uint32_t)(v[j + 1] >= am.y) << (j + 1)) |
                  ((uint32_t)(v[j + 2] >= am.z) << (j + 2)) | ((uint32_t)(v[j + 3] >= am.w) << (j + 3));
          }
        } else {
#pragma unroll
          for (uint32_t j = 0; j < 32; j++) {
            const uint32_t q = cb + j;
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
        while (__any_sync(0xFFFFFFFFu, hm != 0)) {
          const bool has = hm != 0;
          const uint32_t j = has ? (uint32_t)(__ffs(hm) - 1) : 0u;
          const uint32_t bal = __ballot_sync(0xFFFFFFFFu, has);
          const uint32_t pos = wcount + __popc(bal & lt);
          if (has && pos < kPSegCap) {
            uint32_t acc = v[0];
#pragma unroll
            for (uint32_t jj = 1; jj < 32; jj++) acc = jj == j ? v[jj] : acc;
            list[pos] = make_uint2(acc, (cb + j) | (row << 16));
          }
          wcount += __popc(bal);
          hm &= hm - 1;
        }
      }
      // the accumulator is in registers / the list: release it to the MMA
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        if (PAIR)
          arrive_remote(acc_empty0 + 8 * b);
        else
          mbar_arrive(&S.acc_empty[b]);
      }
      if (!dense) {
        // slots within each query's share of the tile, one global atomic per
        // query per tile, then each warp writes its segment
        const uint32_t tot = wcount < kPSegCap ? wcount : kPSegCap;
        if (wcount > kPSegCap && lane == 0) atomicExch(&S.seg_full, 1u);
        __syncwarp();
        for (uint32_t j = lane; j < tot; j += 32) {
          const uint32_t y = list[j].y;
          list[j].y = y | (atom_add_shared(&S.cnt[y & 255], 1u) << 8);  // slot < 256
        }
        epi_sync();
        if (et < nqt) {
          if (S.seg_full)  // some kept doc did not fit: mark every query (bit 31 > cap)
            atomicOr(&a.cnt[q0 + et], 0x80000000u);
          else if (S.cnt[et])
            S.base[et] = atomicAdd(&a.cnt[q0 + et], S.cnt[et]);
        }
        epi_sync();
        for (uint32_t j = lane; j < tot; j += 32) {
          const uint2 en = list[j];
          const uint32_t q = en.y & 255, li = (en.y >> 8) & 255, rw = en.y >> 16;
          const uint32_t pos = S.base[q] + li;
          if (pos < a.cap) {
            a.f_keys[(q0 + q) * a.cap + pos] =
                MODE == 0 ? desc_key(tc_score(en.x, S.bias[q], S.invq[q], a.inv_norm)) : bm_key_q(a, S.qpop[q], en.x);
            const uint64_t rpb = (dt * 8 + rank * (kPRows / 32) + (rw >> 5)) * a.block_stride;
            a.f_ids[(q0 + q) * a.cap + pos] = (uint32_t)(rpb * 32 + (rw & 31));
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (PAIR) cluster_sync_all();  // neither CTA frees the pair's tensor memory while the other uses it
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 1) {
    if (PAIR)
      asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kPTmemCols) : "memory");
    else
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kPTmemCols) : "memory");
  }
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kPThreads, 1)
    fastscan_pair_kernel(const __grid_constant__ CUtensorMap b_map, const TcArgs a, const PairGrid g) {
  pair_body<0, true>(b_map, a, g);
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kPThreads, 1)
    bitmap_pair_kernel(const __grid_constant__ CUtensorMap b_map, const TcArgs a, const PairGrid g) {
  pair_body<1, true>(b_map, a, g);
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kPThreads, 1)
    bitmap_fp4_pair_kernel(const __grid_constant__ CUtensorMap b_map, const TcArgs a, const PairGrid g) {
  pair_body<2, true>(b_map, a, g);
}

__global__ void __launch_bounds__(kPThreads, 1)
    fastscan_persist_kernel(const __grid_constant__ CUtensorMap b_map, const TcArgs a, const PairGrid g) {
  pair_body<0, false>(b_map, a, g);
}

__global__ void __launch_bounds__(kPThreads, 1)
    bitmap_persist_kernel(const __grid_constant__ CUtensorMap b_map, const TcArgs a, const PairGrid g) {
  pair_body<1, false>(b_map, a, g);
}

// clusters of two that can be resident at once (each CTA takes a whole SM)
uint32_t resident_pairs(const void* kernel, size_t smem) {
  static std::mutex mu;
  static int cached[3] = {0, 0, 0};
  const int slot = kernel == (const void*)fastscan_pair_kernel ? 0 : kernel == (const void*)bitmap_pair_kernel ? 1 : 2;
  std::lock_guard<std::mutex> lk(mu);
  if (!cached[slot]) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2, 1, 1);
    cfg.blockDim = dim3(kPThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kernel, &cfg) != cudaSuccess || n < 1) {
      cudaGetLastError();
      int dev = 0, sms = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      n = sms / 2 > 0 ? sms / 2 : 1;
    }
    cached[slot] = n;
  }
  return (uint32_t)cached[slot];
}

}  // namespace

// Which tensor-core scan form a launch uses: OVB_TC_FORM=tile|persist|pair
// forces one (OVB_TC_PAIR=0/1 is tile/pair).  Default: the bitmap family on
// CTA pairs (the one-CTA form is epilogue-bound there: 22 % slower);
// FastScan on the persistent one-CTA form, both being bound by the MMA rate.
TcForm tc_form(int mode) {
  const char* f = getenv("OVB_TC_FORM");
  if (f && f[0]) return f[0] == 't' ? TcForm::kTile : f[1] == 'e' ? TcForm::kPersist : TcForm::kPair;
  const char* e = getenv("OVB_TC_PAIR");
  if (e && e[0] == '0') return TcForm::kTile;
  if (e && e[0] == '1') return TcForm::kPair;
  return mode == 1 ? TcForm::kPair : TcForm::kPersist;
}

// kept entries one epilogue warp of the persistent one-CTA form may hold per tile
uint32_t tc_persist_seg_cap() { return PT<false>::kSegCap; }

// The FP4 form of the bitmap filter takes rows the builders keep whole in
// shared memory.
uint32_t tc_fp4_max_words() { return kPRowCacheWords; }

template <int MODE>
void launch_tc_pair(TcArgs a, const uint8_t* b_rows, cudaStream_t stream, bool pair) {
  if (!a.n || !a.nq) return;
  if (pair && a.nq > kPMaxQ) {
    // the pair form stages every query's parameters in shared memory: launch
    // query chunks of at most kPMaxQ
    const uint64_t k_bytes = (uint64_t)a.n_kb * kPKBytes;
    for (uint64_t q0 = 0; q0 < a.nq; q0 += kPMaxQ) {
      TcArgs c = a;
      c.nq = a.nq - q0 < kPMaxQ ? a.nq - q0 : kPMaxQ;
      if (c.qpop) c.qpop += q0;
      if (c.bias) c.bias += q0;
      if (c.invq) c.invq += q0;
      if (c.keys) c.keys += q0 * a.ld;
      if (c.thr) c.thr += q0 * a.thr_stride;
      if (c.thr_pos) c.thr_pos += q0 * a.thr_stride;
      if (c.cnt) c.cnt += q0;
      if (c.f_keys) c.f_keys += q0 * a.cap;
      if (c.f_ids) c.f_ids += q0 * a.cap;
      launch_tc_pair<MODE>(c, b_rows + q0 * k_bytes, stream, pair);
    }
    return;
  }
  const char* what = MODE == 0 ? "FastScan tensor-core scan" : MODE == 1 ? "bitmap tensor-core scan"
                                                                          : "bitmap FP4 tensor-core scan";
  const uint64_t k_bytes = (uint64_t)a.n_kb * kPKBytes;
  if (!a.n_kb || (MODE == 0 && a.n_kb % 4)) throw std::invalid_argument(std::string(what) + ": bad K extent");
  if (MODE == 2) {
    // query tiles of at most kPF4TileN columns (OVB_FP4_TILE_N: 16..224), balanced: a multiple of 16
    if (!pair || a.keys || a.qpv > kPRowCacheWords || 4ull * a.n_kb < a.qpv)
      throw std::invalid_argument(std::string(what) + ": needs CTA pairs, a filter and rows of <= 16 words");
    uint32_t tile_n = kPF4TileN;
    if (const char* e = getenv("OVB_FP4_TILE_N")) {
      const long v = strtol(e, nullptr, 10);
      if (v >= 16 && v <= (long)kPF4MaxN) tile_n = (uint32_t)(v / 16 * 16);
    }
    const uint64_t qt = (a.nq + tile_n - 1) / tile_n;
    a.nt = (uint32_t)(((a.nq + qt - 1) / qt + 15) / 16 * 16);
  } else {
    a.nt = a.nq >= kPMaxN ? kPMaxN : (uint32_t)((a.nq + 15) / 16 * 16);  // a multiple of 16 in [16, 256]
  }
  CUtensorMap map;
  cuuint64_t gdim[2] = {(cuuint64_t)k_bytes, (cuuint64_t)a.nq};
  cuuint64_t gstride[1] = {(cuuint64_t)k_bytes};
  cuuint32_t box[2] = {(cuuint32_t)kPKBytes, (cuuint32_t)(pair ? a.nt / 2 : a.nt)};
  cuuint32_t estride[2] = {1, 1};
  CUresult rc = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)b_rows, gdim, gstride, box, estride,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rc != CUDA_SUCCESS) throw CudaError(std::string("cuTensorMapEncodeTiled failed: ") + what);
  if (MODE == 0 && 255ull * a.pairs_pad >= (1ull << 23)) throw std::invalid_argument(std::string(what) + ": dim too large");
  if (MODE == 1 && (64ull * a.qpv >= (1ull << 24) || 2ull * a.n_kb < a.qpv))
    throw std::invalid_argument(std::string(what) + ": row too long");
  if (MODE == 2 && 64ull * a.qpv >= (1ull << 23)) throw std::invalid_argument(std::string(what) + ": row too long");
  if (!a.keys && a.block_stride != 1) throw std::invalid_argument(std::string(what) + ": filter needs stride 1");
  const uint64_t n_blocks = (a.n + 31) / 32;
  const uint64_t logical_blocks = (n_blocks + a.block_stride - 1) / a.block_stride;
  PairGrid g;
  const uint64_t doc_tiles = (logical_blocks + 7) / 8;
  const uint64_t q_tiles = (a.nq + a.nt - 1) / a.nt;
  if (doc_tiles * q_tiles + 2048 > 0xFFFFFFFFull || a.n >= (1ull << 32))
    throw std::invalid_argument(std::string(what) + ": too many tiles; split the query batch");
  g.n_doc_tiles = (uint32_t)doc_tiles;
  g.q_tiles = (uint32_t)q_tiles;
  const uint64_t total = doc_tiles * q_tiles;
  if (pair) {
    auto kernel = MODE == 0 ? fastscan_pair_kernel : MODE == 1 ? bitmap_pair_kernel : bitmap_fp4_pair_kernel;
    const size_t smem = sizeof(PSmem<true>) + 1024;
    OVB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    uint64_t clusters = resident_pairs((const void*)kernel, smem);
    // whole doc tiles per cluster once every cluster gets at least two of them
    g.doc_major = doc_tiles >= 2 * clusters ? 1u : 0u;
    if (clusters > total) clusters = total;
    kernel<<<(unsigned)(2 * clusters), kPThreads, smem, stream>>>(map, a, g);
  } else if constexpr (MODE != 2) {
    auto kernel = MODE == 0 ? fastscan_persist_kernel : bitmap_persist_kernel;
    const size_t smem = sizeof(PSmem<false>) + 1024;
    OVB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 0;
    OVB_CUDA(cudaGetDevice(&dev));
    OVB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    uint64_t ctas = (uint64_t)sms;  // one CTA per SM (its shared memory and TMEM fill the SM)
    g.doc_major = 0;
    if (ctas > total) ctas = total;
    kernel<<<(unsigned)ctas, kPThreads, smem, stream>>>(map, a, g);
  }
  launched();
}

template void launch_tc_pair<0>(TcArgs, const uint8_t*, cudaStream_t, bool);
template void launch_tc_pair<1>(TcArgs, const uint8_t*, cudaStream_t, bool);
template void launch_tc_pair<2>(TcArgs, const uint8_t*, cudaStream_t, bool);

}  // namespace ovb
