// K7: exact, deterministic per-row top-k selection.
//
// Reproduces the reference's composite-key selection contract -- TopK
// (src/util.rs:375-600), select_nth_unstable_by + head sort on
// (score, doc_id) (src/sign_bitmap.rs:350-361, src/bitmap.rs:281-289) and the
// ABI's normalize_global_order (ordvec-ffi/src/lib.rs:430-435) -- as a radix
// select over the logical 64-bit key (key32 << 32) | id32, smaller is better.
// Keys with equal (score, id) (duplicate candidate rows) are interchangeable:
// any `need` of them give identical output, so no slot order is required.
//
// One CTA per row.  Per digit (11 bits at a time, most significant first,
// skipping bits that are zero in every key) the CTA histograms the keys that
// still match the fixed prefix, finds the bin holding the k-th key, and stops
// as soon as that bin holds exactly the keys still needed.  A collect pass
// then gathers the k winners and a bitonic sort orders them.
#include <cooperative_groups.h>

#include "ovb_common.cuh"
#include "ovb_kernels.h"

namespace ovb {

namespace {

constexpr int kSelThreads = 1024;
constexpr int kHistBins = 2048;
constexpr uint64_t kShortRow = 16384;  // rows up to this many keys take the 256-thread form
constexpr uint32_t kShortCap = 2048;   // ... when k is at most this

struct Digit {
  uint32_t shift, width;
};

__device__ __forceinline__ uint64_t load_key(const uint32_t* keys, const uint32_t* ids,
                                             uint64_t i) {
  uint32_t k = keys[i];
  uint32_t id = ids ? ids[i] : (uint32_t)i;
  return ((uint64_t)k << 32) | id;
}

// In-place bitonic sort of buf[0..len) ascending, len a power of two.
__device__ void bitonic_sort(uint64_t* buf, uint32_t len) {
  for (uint32_t size = 2; size <= len; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t t = threadIdx.x; t < len / 2; t += blockDim.x) {
        uint32_t i = 2 * t - (t & (stride - 1));
        uint32_t j = i + stride;
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
}

// T threads per row (1024; 256 for rows of at most kShortRow keys, so that
// several rows share an SM), CAP sorted entries in shared memory.
template <int T, uint32_t CAP>
__global__ void __launch_bounds__(T)
    select_rows_kernel(SelectArgs a, uint64_t* gbuf, uint32_t gbuf_stride) {
  constexpr int BPT = kHistBins / T;  // histogram bins per thread in the scan
  __shared__ uint32_t hist[kHistBins];
  __shared__ uint32_t warp_tot[T / 32];
  __shared__ uint64_t sbuf[CAP];
  __shared__ uint32_t s_bin, s_before, s_in_bin, s_cnt_below, s_cnt_tie;

  const uint64_t row = blockIdx.x;
  uint64_t start, n;
  if (a.row_off) {
    start = a.row_off[row];
    n = a.row_off[row + 1] - start;
  } else {
    start = row * a.ld;
    n = a.n;
    if (a.row_len && a.row_len[row] < n) n = a.row_len[row];
  }
  const uint32_t* keys = a.keys + start;
  const uint32_t* ids = a.ids ? a.ids + start : nullptr;
  const uint32_t k_eff = (uint32_t)(n < a.k ? n : a.k);
  uint32_t* out_k = a.out_keys + row * (uint64_t)a.k;
  uint32_t* out_i = a.out_ids + row * (uint64_t)a.k;

  for (uint32_t j = k_eff + threadIdx.x; j < a.k; j += blockDim.x) {
    out_k[j] = kSentinelKey;
    out_i[j] = kSentinelId;
  }
  if (k_eff == 0) return;

  uint64_t* buf = (k_eff <= CAP) ? sbuf : gbuf + row * (uint64_t)gbuf_stride;

  // digit schedule: key32 bits [32+key_bits-1, 32], then id bits [id_bits-1, 0]
  Digit digits[8];
  int nd = 0;
  for (int part = 0; part < 2; part++) {
    uint32_t bits = part == 0 ? a.key_bits : a.id_bits;
    uint32_t top = (part == 0 ? 32u : 0u) + bits;
    while (bits > 0) {
      uint32_t w = bits < 11 ? bits : 11;
      top -= w;
      digits[nd++] = Digit{top, w};
      bits -= w;
    }
  }

  uint64_t prefix = 0, fixed = 0;
  uint32_t need = k_eff;
  bool take_all = (k_eff == n);
  for (int d = 0; d < nd && !take_all; d++) {
    const uint32_t shift = digits[d].shift, width = digits[d].width;
    const uint32_t nbins = 1u << width;
    for (uint32_t b = threadIdx.x; b < kHistBins; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
      uint64_t key = load_key(keys, ids, i);
      if ((key & fixed) == prefix) atomicAdd(&hist[(uint32_t)(key >> shift) & (nbins - 1)], 1u);
    }
    __syncthreads();
    // block scan over bins (BPT consecutive bins per thread) to find the bin
    // holding the need-th key
    const uint32_t t = threadIdx.x;
    uint32_t hv[BPT];
    uint32_t s = 0;
#pragma unroll
    for (int b = 0; b < BPT; b++) {
      hv[b] = hist[BPT * t + b];
      s += hv[b];
    }
    uint32_t incl = s;
    const int lane = t & 31, w = t >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
      uint32_t v = lane < T / 32 ? warp_tot[lane] : 0u, x = v;
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
      }
      if (lane < T / 32) warp_tot[lane] = x - v;  // exclusive warp offsets
    }
    __syncthreads();
    const uint32_t excl = warp_tot[w] + incl - s;
    if (excl < need && need <= excl + s) {
      uint32_t before = excl;
#pragma unroll
      for (int b = 0; b < BPT; b++) {
        if (need <= before + hv[b]) {
          s_bin = BPT * t + b;
          s_before = before;
          s_in_bin = hv[b];
          break;
        }
        before += hv[b];
      }
    }
    __syncthreads();
    need -= s_before;
    prefix |= (uint64_t)s_bin << shift;
    fixed |= (uint64_t)(nbins - 1) << shift;
    if (s_in_bin == need) take_all = true;  // the whole bin is taken
    __syncthreads();
  }

  // collect: keys strictly below the prefix, then `need` keys inside it
  if (threadIdx.x == 0) {
    s_cnt_below = 0;
    s_cnt_tie = 0;
  }
  __syncthreads();
  const uint32_t below_total = k_eff - need;
  for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
    uint64_t key = load_key(keys, ids, i);
    uint64_t m = key & fixed;
    if (m < prefix) {
      uint32_t slot = atomicAdd(&s_cnt_below, 1u);
      if (slot < below_total) buf[slot] = key;
    } else if (m == prefix) {
      uint32_t tk = atomicAdd(&s_cnt_tie, 1u);
      if (tk < need) buf[below_total + tk] = key;
    }
  }
  __syncthreads();
  if (!a.unordered) {  // a caller that needs only the set skips the sort
    uint32_t len = 1;
    while (len < k_eff) len <<= 1;
    for (uint32_t j = k_eff + threadIdx.x; j < len; j += blockDim.x) buf[j] = ~0ull;
    __syncthreads();
    bitonic_sort(buf, len);
  }
  for (uint32_t j = threadIdx.x; j < k_eff; j += blockDim.x) {
    uint64_t key = buf[j];
    out_k[j] = (uint32_t)(key >> 32);
    out_i[j] = (uint32_t)key;
  }
}

// Cluster form for few long rows (the one-query-per-launch path): a cluster of
// kClusterCtas CTAs shares one row.  Each CTA histograms its contiguous slice;
// the per-CTA histograms are summed through distributed shared memory, every
// CTA derives the same bin, and the winners are gathered into CTA 0's shared
// memory, which sorts and writes them.  All waits are hardware cluster
// barriers.  When a CTA's slice fits (stage != 0) it is first copied into
// dynamic shared memory (keys, and explicit ids) with several loads in flight
// per thread, and every pass reads it there: the passes are otherwise bound by
// the latency of re-reading the slice from L2.
constexpr int kClusterCtas = 8;
constexpr uint32_t kClusterCap = 2048;
constexpr uint64_t kClusterStageBytes = 160 * 1024;

__global__ void __cluster_dims__(kClusterCtas, 1, 1) __launch_bounds__(kSelThreads)
    select_rows_cluster_kernel(SelectArgs a, uint32_t stage) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  __shared__ uint32_t hist[kHistBins];
  __shared__ uint32_t tot[kHistBins];
  __shared__ uint32_t warp_tot[kSelThreads / 32];
  __shared__ uint64_t sbuf[kClusterCap];
  __shared__ uint32_t s_bin, s_before, s_in_bin, s_cnt_below, s_cnt_tie, s_ctie;

  const uint32_t crank = cluster.block_rank();
  const uint64_t row = blockIdx.x / kClusterCtas;
  uint64_t start, n;
  if (a.row_off) {
    start = a.row_off[row];
    n = a.row_off[row + 1] - start;
  } else {
    start = row * a.ld;
    n = a.n;
  }
  const uint32_t* keys = a.keys + start;
  const uint32_t* ids = a.ids ? a.ids + start : nullptr;
  const uint32_t k_eff = (uint32_t)(n < a.k ? n : a.k);
  const uint64_t per = (n + kClusterCtas - 1) / kClusterCtas;
  const uint64_t lo = crank * per < n ? crank * per : n;
  const uint64_t hi = lo + per < n ? lo + per : n;
  extern __shared__ __align__(16) uint32_t st_keys[];  // [per] keys, then [per] ids when explicit
  uint32_t* st_ids = st_keys + per;
  // Stage the slice once, eight loads in flight per thread (one pass of
  // dependent loads would wait out the memory latency once per key).
  if (stage) {
    for (uint64_t i0 = lo + threadIdx.x; i0 < hi; i0 += 8ull * blockDim.x) {
      uint32_t v[8], u[8];
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const uint64_t i = i0 + (uint64_t)j * blockDim.x;
        v[j] = i < hi ? keys[i] : 0u;
        u[j] = i < hi && ids ? ids[i] : 0u;
      }
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const uint64_t i = i0 + (uint64_t)j * blockDim.x;
        if (i < hi) {
          st_keys[i - lo] = v[j];
          if (ids) st_ids[i - lo] = u[j];
        }
      }
    }
    __syncthreads();
  }
  // key i of this CTA's slice
  auto key_at = [&](uint64_t i) -> uint64_t {
    if (!stage) return load_key(keys, ids, i);
    return ((uint64_t)st_keys[i - lo] << 32) | (ids ? st_ids[i - lo] : (uint32_t)i);
  };

  // Digits of key32 and, for explicit ids, of the id.  When the id is the
  // position (ids == null), ties left after the key digits are resolved by
  // position instead: the CTAs' slices are ordered, so the lowest positions are
  // the first CTAs' ties in slice order (two passes fewer).
  Digit digits[8];
  int nd = 0;
  for (int part = 0; part < (ids ? 2 : 1); part++) {
    uint32_t bits = part == 0 ? a.key_bits : a.id_bits;
    uint32_t top = (part == 0 ? 32u : 0u) + bits;
    while (bits > 0) {
      uint32_t w = bits < 11 ? bits : 11;
      top -= w;
      digits[nd++] = Digit{top, w};
      bits -= w;
    }
  }

  uint64_t prefix = 0, fixed = 0;
  uint32_t need = k_eff;
  bool take_all = (k_eff == n);
  for (int d = 0; d < nd && !take_all && k_eff > 0; d++) {
    const uint32_t shift = digits[d].shift, width = digits[d].width;
    const uint32_t nbins = 1u << width;
    for (uint32_t b = threadIdx.x; b < kHistBins; b += blockDim.x) hist[b] = 0;
    cluster.sync();
    for (uint64_t i0 = lo + threadIdx.x; i0 < hi; i0 += 4ull * blockDim.x) {  // four keys in flight
      uint64_t kk[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const uint64_t i = i0 + (uint64_t)j * blockDim.x;
        kk[j] = i < hi ? key_at(i) : 0;
      }
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (i0 + (uint64_t)j * blockDim.x < hi && (kk[j] & fixed) == prefix)
          atomicAdd(&hist[(uint32_t)(kk[j] >> shift) & (nbins - 1)], 1u);
    }
    cluster.sync();
    for (uint32_t b = threadIdx.x; b < kHistBins; b += blockDim.x) {
      uint32_t s = 0;
      for (int r = 0; r < kClusterCtas; r++) s += cluster.map_shared_rank(hist, r)[b];
      tot[b] = s;
    }
    __syncthreads();
    const uint32_t t = threadIdx.x;
    uint32_t h0 = tot[2 * t], h1 = tot[2 * t + 1];
    uint32_t s = h0 + h1, incl = s;
    const int lane = t & 31, w = t >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
      uint32_t v = warp_tot[lane], x = v;
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
      }
      warp_tot[lane] = x - v;
    }
    __syncthreads();
    uint32_t excl = warp_tot[w] + incl - s;
    if (excl < need && need <= excl + s) {
      if (need <= excl + h0) {
        s_bin = 2 * t;
        s_before = excl;
        s_in_bin = h0;
      } else {
        s_bin = 2 * t + 1;
        s_before = excl + h0;
        s_in_bin = h1;
      }
    }
    __syncthreads();
    need -= s_before;
    prefix |= (uint64_t)s_bin << shift;
    fixed |= (uint64_t)(nbins - 1) << shift;
    if (s_in_bin == need) take_all = true;
    // no CTA may reset its histogram while another still reads it
    cluster.sync();
  }

  uint32_t* out_k = a.out_keys + row * (uint64_t)a.k;
  uint32_t* out_i = a.out_ids + row * (uint64_t)a.k;
  if (crank == 0) {
    for (uint32_t j = k_eff + threadIdx.x; j < a.k; j += blockDim.x) {
      out_k[j] = kSentinelKey;
      out_i[j] = kSentinelId;
    }
    if (threadIdx.x == 0) {
      s_cnt_below = 0;
      s_cnt_tie = 0;
    }
  }
  cluster.sync();
  const uint32_t below_total = k_eff - need;
  uint64_t* buf0 = cluster.map_shared_rank(sbuf, 0);
  uint32_t* below0 = cluster.map_shared_rank(&s_cnt_below, 0);
  uint32_t* tie0 = cluster.map_shared_rank(&s_cnt_tie, 0);
  // more ties than needed and ids are positions: take the lowest positions
  const bool by_pos = !ids && !take_all && k_eff > 0;
  if (k_eff > 0) {
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
      uint64_t key = key_at(i);
      uint64_t m = key & fixed;
      if (m < prefix) {
        uint32_t slot = atomicAdd(below0, 1u);
        if (slot < below_total) buf0[slot] = key;
      } else if (m == prefix && !by_pos) {
        uint32_t tk = atomicAdd(tie0, 1u);
        if (tk < need) buf0[below_total + tk] = key;
      }
    }
  }
  if (by_pos) {
    // each thread owns a contiguous run of the slice: count its ties, scan the
    // counts over the CTA, add the ties of the lower-ranked CTAs, then write
    // the ties whose rank falls below `need` at that rank
    const uint64_t run = (hi - lo + blockDim.x - 1) / blockDim.x;
    const uint64_t r0 = lo + threadIdx.x * run < hi ? lo + threadIdx.x * run : hi;
    const uint64_t r1 = r0 + run < hi ? r0 + run : hi;
    uint32_t mine = 0;
    for (uint64_t i = r0; i < r1; i++) mine += (key_at(i) & fixed) == prefix ? 1u : 0u;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
      const uint32_t v = warp_tot[lane];
      uint32_t x = v;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
      }
      warp_tot[lane] = x - v;
      if (lane == 31) s_ctie = x;
    }
    __syncthreads();
    uint32_t rank = warp_tot[w] + incl - mine;
    cluster.sync();  // every CTA's s_ctie is set
    for (uint32_t r = 0; r < crank; r++) rank += *cluster.map_shared_rank(&s_ctie, r);
    for (uint64_t i = r0; i < r1 && rank < need; i++) {
      const uint64_t key = key_at(i);
      if ((key & fixed) == prefix) buf0[below_total + rank++] = key;
    }
  }
  cluster.sync();
  if (crank == 0 && k_eff > 0) {
    if (!a.unordered) {
      uint32_t len = 1;
      while (len < k_eff) len <<= 1;
      for (uint32_t j = k_eff + threadIdx.x; j < len; j += blockDim.x) sbuf[j] = ~0ull;
      __syncthreads();
      bitonic_sort(sbuf, len);
    }
    for (uint32_t j = threadIdx.x; j < k_eff; j += blockDim.x) {
      out_k[j] = (uint32_t)(sbuf[j] >> 32);
      out_i[j] = (uint32_t)sbuf[j];
    }
  }
}

// Whole-GPU form for a few very long rows (one query per call over millions
// of docs): each digit pass is one launch whose CTAs histogram grid-stride
// slices of every row into a global histogram; the last CTA of a row to
// finish (atomic arrival count after a fence) scans it, fixes the digit and
// resets the histogram.  A collect launch gathers the winners the same way and
// its last CTA per row sorts and writes them.  No CTA waits for another.
constexpr uint32_t kWideRows = 16;
constexpr uint64_t kWideMinN = 1u << 20;
constexpr int kWideThreads = 512;

struct WideState {
  uint64_t prefix, fixed;
  uint32_t need, done, arrive, below, tie, pad;
};
static_assert(sizeof(WideState) == 40, "WideState layout");

struct WideScratch {
  uint32_t* hist;    // rows x kHistBins
  WideState* state;  // rows
  uint64_t* win;     // rows x k
};

__host__ __device__ inline uint64_t wide_state_elems(uint64_t rows) { return (rows * sizeof(WideState) + 7) / 8; }

__host__ inline WideScratch wide_scratch(uint64_t* scratch, uint64_t rows) {
  WideScratch w;
  w.hist = reinterpret_cast<uint32_t*>(scratch);
  w.state = reinterpret_cast<WideState*>(scratch + rows * (kHistBins / 2));
  w.win = scratch + rows * (kHistBins / 2) + wide_state_elems(rows);
  return w;
}

__global__ void wide_init_kernel(SelectArgs a, WideScratch w) {
  const uint64_t row = blockIdx.x;
  for (uint32_t b = threadIdx.x; b < kHistBins; b += blockDim.x) w.hist[row * kHistBins + b] = 0;
  if (threadIdx.x == 0) {
    WideState& st = w.state[row];
    st.prefix = 0;
    st.fixed = 0;
    st.need = (uint32_t)(a.n < a.k ? a.n : a.k);
    st.done = st.need == a.n;  // every key is a winner
    st.arrive = st.below = st.tie = st.pad = 0;
  }
}

// Exclusive scan of hist[0..kHistBins) by kWideThreads threads (4 bins each);
// the thread whose bins hold the need-th key writes (bin, before, in_bin).
__device__ void wide_find_bin(const uint32_t* hist, uint32_t need, uint32_t* out3) {
  __shared__ uint32_t warp_tot[kWideThreads / 32];
  const uint32_t t = threadIdx.x, lane = t & 31, wp = t >> 5;
  uint32_t h[4], sum = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    h[j] = hist[4 * t + j];
    sum += h[j];
  }
  uint32_t incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_tot[wp] = incl;
  __syncthreads();
  if (wp == 0) {
    const uint32_t v = lane < kWideThreads / 32 ? warp_tot[lane] : 0;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if (lane >= o) x += y;
    }
    if (lane < kWideThreads / 32) warp_tot[lane] = x - v;
  }
  __syncthreads();
  uint32_t before = warp_tot[wp] + incl - sum;
  if (before < need && need <= before + sum) {
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (need <= before + h[j]) {
        out3[0] = 4 * t + j;
        out3[1] = before;
        out3[2] = h[j];
        break;
      }
      before += h[j];
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kWideThreads) wide_hist_kernel(SelectArgs a, WideScratch w, uint32_t shift,
                                                                 uint32_t width) {
  __shared__ uint32_t hist[kHistBins];
  __shared__ uint32_t s_last, s_pick[3];
  const uint64_t row = blockIdx.y;
  WideState& st = w.state[row];
  if (*reinterpret_cast<volatile uint32_t*>(&st.done)) return;  // uniform per row
  const uint64_t prefix = st.prefix, fixed = st.fixed;
  const uint32_t mask = (1u << width) - 1;
  for (uint32_t b = threadIdx.x; b < kHistBins; b += blockDim.x) hist[b] = 0;
  __syncthreads();
  const uint32_t* keys = a.keys + row * a.ld;
  const uint32_t* ids = a.ids ? a.ids + row * a.ld : nullptr;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t key = load_key(keys, ids, i);
    if ((key & fixed) == prefix) atomicAdd(&hist[(uint32_t)(key >> shift) & mask], 1u);
  }
  __syncthreads();
  uint32_t* gh = w.hist + row * kHistBins;
  for (uint32_t b = threadIdx.x; b <= mask; b += blockDim.x)
    if (hist[b]) atomicAdd(&gh[b], hist[b]);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&st.arrive, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  // last CTA of this row: every other CTA's histogram is in gh
  __threadfence();
  for (uint32_t b = threadIdx.x; b < kHistBins; b += blockDim.x) {
    hist[b] = b <= mask ? *reinterpret_cast<volatile uint32_t*>(&gh[b]) : 0u;
    gh[b] = 0;
  }
  __syncthreads();
  const uint32_t need = st.need;
  wide_find_bin(hist, need, s_pick);
  if (threadIdx.x == 0) {
    st.need = need - s_pick[1];
    st.prefix = prefix | ((uint64_t)s_pick[0] << shift);
    st.fixed = fixed | ((uint64_t)mask << shift);
    st.done = s_pick[2] == need - s_pick[1];  // the whole bin is taken
    st.arrive = 0;
  }
}

// Collect: keys strictly below the prefix, then `need` keys inside it; the last
// CTA of a row sorts the k winners and writes them.
__global__ void __launch_bounds__(kWideThreads) wide_collect_kernel(SelectArgs a, WideScratch w) {
  __shared__ uint64_t buf[kSelectSmemCap];
  __shared__ uint32_t s_last;
  const uint64_t row = blockIdx.y;
  WideState& st = w.state[row];
  const uint64_t prefix = st.prefix, fixed = st.fixed;
  const uint32_t k_eff = (uint32_t)(a.n < a.k ? a.n : a.k), need = st.need;
  const uint32_t below_total = k_eff - need;
  const uint32_t* keys = a.keys + row * a.ld;
  const uint32_t* ids = a.ids ? a.ids + row * a.ld : nullptr;
  uint64_t* win = w.win + row * (uint64_t)a.k;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  // warp-uniform trip count so the ballots see every lane
  const uint64_t first = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
  for (uint64_t base = first; base < a.n; base += stride) {
    const uint64_t i = base + lane;
    uint64_t key = 0;
    bool lo = false, eq = false;
    if (i < a.n) {
      key = load_key(keys, ids, i);
      const uint64_t m = key & fixed;
      lo = m < prefix;
      eq = m == prefix;
    }
    uint32_t lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    const uint32_t bl = __ballot_sync(0xFFFFFFFFu, lo), be = __ballot_sync(0xFFFFFFFFu, eq);
    uint32_t b0 = 0, e0 = 0;
    if (lane == 0) {
      if (bl) b0 = atomicAdd(&st.below, (uint32_t)__popc(bl));
      if (be) e0 = atomicAdd(&st.tie, (uint32_t)__popc(be));
    }
    b0 = __shfl_sync(0xFFFFFFFFu, b0, 0);
    e0 = __shfl_sync(0xFFFFFFFFu, e0, 0);
    if (lo) {
      const uint32_t slot = b0 + __popc(bl & lt);
      if (slot < below_total) win[slot] = key;
    } else if (eq) {
      const uint32_t slot = e0 + __popc(be & lt);
      if (slot < need) win[below_total + slot] = key;
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&st.arrive, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  uint32_t len = 1;
  while (len < k_eff) len <<= 1;
  for (uint32_t j = threadIdx.x; j < len; j += blockDim.x)
    buf[j] = j < k_eff ? *reinterpret_cast<volatile uint64_t*>(&win[j]) : ~0ull;
  __syncthreads();
  bitonic_sort(buf, len);
  uint32_t* out_k = a.out_keys + row * (uint64_t)a.k;
  uint32_t* out_i = a.out_ids + row * (uint64_t)a.k;
  for (uint32_t j = threadIdx.x; j < a.k; j += blockDim.x) {
    out_k[j] = j < k_eff ? (uint32_t)(buf[j] >> 32) : kSentinelKey;
    out_i[j] = j < k_eff ? (uint32_t)buf[j] : kSentinelId;
  }
}

void launch_select_wide(const SelectArgs& a, uint64_t rows, uint64_t* scratch, cudaStream_t stream) {
  const WideScratch w = wide_scratch(scratch, rows);
  wide_init_kernel<<<(unsigned)rows, 256, 0, stream>>>(a, w);
  uint64_t per_row = (a.n + kWideThreads * 32 - 1) / (kWideThreads * 32);  // ~32 keys per thread
  const uint64_t cap = (148ull * 4 + rows - 1) / rows;
  if (per_row > cap) per_row = cap;
  if (per_row < 1) per_row = 1;
  const dim3 grid((unsigned)per_row, (unsigned)rows);
  for (int part = 0; part < 2; part++) {  // key bits, then id bits, 11 at a time from the top
    uint32_t bits = part == 0 ? a.key_bits : a.id_bits;
    uint32_t top = (part == 0 ? 32u : 0u) + bits;
    while (bits > 0) {
      const uint32_t wd = bits < 11 ? bits : 11;
      top -= wd;
      wide_hist_kernel<<<grid, kWideThreads, 0, stream>>>(a, w, top, wd);
      bits -= wd;
    }
  }
  wide_collect_kernel<<<grid, kWideThreads, 0, stream>>>(a, w);
  launched();
}

bool use_select_wide(const SelectArgs& a, uint64_t rows, const uint64_t* scratch) {
  return scratch && !a.row_off && !a.row_len && rows <= kWideRows && a.n >= kWideMinN && a.k <= kSelectSmemCap;
}

}  // namespace

size_t select_rows_scratch_elems(uint64_t rows, uint32_t k, uint64_t n) {
  uint64_t len = 1;
  while (len < k) len <<= 1;
  uint64_t e = k <= kSelectSmemCap ? 0 : rows * len;
  if (rows <= kWideRows && k <= kSelectSmemCap && n >= kWideMinN) {  // the whole-GPU form for few long rows
    const uint64_t wide = rows * (kHistBins / 2) + wide_state_elems(rows) + rows * (uint64_t)k;
    if (wide > e) e = wide;
  }
  return e;
}

void launch_select_rows(const SelectArgs& a, uint64_t rows, uint64_t* scratch,
                        cudaStream_t stream) {
  if (rows == 0) return;
  const char* wide_env = getenv("OVB_SELECT_WIDE");  // "0" keeps the cluster / per-row forms
  if (!(wide_env && wide_env[0] == '0') && use_select_wide(a, rows, scratch)) {
    launch_select_wide(a, rows, scratch, stream);
    return;
  }
  // few long rows: one 8-CTA cluster per row (below two rows per SM the
  // per-row form leaves SMs idle, and one CTA alone streams a long row slowly)
  if (!a.row_off && !a.row_len && a.k <= kClusterCap && a.n >= 32768 &&
      (rows * kClusterCtas <= 2 * 148 || (a.n >= (1ull << 18) && rows < 2 * 148))) {
    const uint64_t per = (a.n + kClusterCtas - 1) / kClusterCtas;
    const uint64_t bytes = per * (a.ids ? 8 : 4);
    const uint32_t stage = bytes <= kClusterStageBytes ? 1u : 0u;
    const size_t smem = stage ? (size_t)bytes : 0;
    if (smem) allow_dynamic_smem(select_rows_cluster_kernel);  // static 32 KiB + the stage
    select_rows_cluster_kernel<<<(unsigned)(rows * kClusterCtas), kSelThreads, smem, stream>>>(a, stage);
    launched();
    return;
  }
  // short uniform rows: 256 threads per row, several rows per SM
  if (!a.row_off && a.n <= kShortRow && a.k <= kShortCap) {
    select_rows_kernel<256, kShortCap><<<(unsigned)rows, 256, 0, stream>>>(a, nullptr, 0);
    launched();
    return;
  }
  uint32_t stride = 0;
  if (a.k > kSelectSmemCap) {
    uint64_t len = 1;
    while (len < a.k) len <<= 1;
    stride = (uint32_t)len;
  }
  select_rows_kernel<kSelThreads, kSelectSmemCap><<<(unsigned)rows, kSelThreads, 0, stream>>>(a, scratch, stride);
  launched();
}

}  // namespace ovb
