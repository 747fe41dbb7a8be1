// Allocation-free variant of the RankQuant full asymmetric search.
//
// Some callers cannot let a library call cudaMalloc: a serving thread with a
// hard latency budget (cudaMalloc/cudaFree can synchronise the whole device),
// or a process whose device memory is owned by one framework allocator with a
// fixed budget, where any allocation made behind that allocator's back breaks
// its accounting.  ovb_rankquant_search_noalloc serves them: the caller passes
// device inputs and outputs, and every intermediate buffer (normalised
// queries, the per-query score keys, the selected top-k keys) is carved out of
// one file-scope device array, g_noalloc_scratch, of fixed size
// kNoAllocScratchBytes (32 MiB).  That array is part of this library's device
// image, so every GPU that loads the library holds it until the process exits.
//
// Host code must not pass the symbol itself to a kernel: on the host,
// `g_noalloc_scratch` names a host-side stand-in, not device memory.  The
// device address is obtained once per device with cudaGetSymbolAddress while
// that device is current; the first call on each device does this set-up, so
// that first call should come before any stream capture.
//
// The cached address belongs to the device context it was looked up in: after
// cudaDeviceReset the next call would reuse a stale address, so this entry
// point must not be used across a device reset.
//
// Every call shares the array and it keeps the last call's contents.  Nothing
// in it needs to start at zero: each byte a call reads is written earlier in
// the same call.  Calls whose work overlaps on the GPU (different streams, or
// different host threads) race on the array; serialise them.
//
// Queries are not checked for finiteness here (that check needs a device to
// host read, i.e. a synchronisation); the caller passes finite queries, and
// the ranking of a non-finite query is unspecified.
#include <cmath>
#include <functional>
#include <mutex>

#include "ovb_host.h"

namespace ovb {
namespace {

constexpr size_t kNoAllocScratchBytes = 32ull << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (set-up once).
uint8_t* scratch_base() {
  int dev = 0;
  OVB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) fail(ORDVEC_STATUS_INTERNAL, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      fail(ORDVEC_STATUS_INTERNAL, std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") +
                                       cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  return (uint8_t*)g_scratch_addr[dev];
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// a * b * c in 64 bits, or false when the product does not fit.
bool mul3(uint64_t a, uint64_t b, uint64_t c, uint64_t* out) {
  uint64_t ab = 0;
  return !__builtin_mul_overflow(a, b, &ab) && !__builtin_mul_overflow(ab, c, out);
}

}  // namespace
}  // namespace ovb

namespace ovb {
// status/last-error boundary of the C ABI (capi.cu)
ordvec_status_t api_boundary(const std::function<void()>& f);
}  // namespace ovb

using namespace ovb;

extern "C" ordvec_status_t ovb_rankquant_search_noalloc(const ordvec_index_t* rq, const float* d_queries,
                                                        uint64_t nq, uint64_t k, float* d_scores,
                                                        int64_t* d_ids, void* stream) {
  return api_boundary([&] {
    ensure_device();
    const Index& ix = as_index(rq);
    if (ix.kind != ORDVEC_INDEX_KIND_RANK_QUANT)
      fail(ORDVEC_STATUS_UNSUPPORTED_OPERATION, "ovb_rankquant_search_noalloc needs a RankQuant index");
    if (nq && !d_queries) fail(ORDVEC_STATUS_NULL_POINTER, "queries pointer is NULL");
    const uint64_t ke = k < ix.n ? k : ix.n;
    if (!ke || !nq) return;
    if (!d_scores || !d_ids) fail(ORDVEC_STATUS_NULL_POINTER, "output pointer is NULL");
    if (ke > kSelectSmemCap)
      fail(ORDVEC_STATUS_BAD_ARGUMENT, "ovb_rankquant_search_noalloc supports k <= 4096");
    // each part is checked for 64-bit overflow and against the array size
    // before it is rounded and summed, so a huge nq cannot wrap the total
    uint64_t parts[3];
    const bool fits = mul3(nq, ix.dim, 4, &parts[0]) && mul3(nq, ix.n, 4, &parts[1]) &&
                      mul3(nq, ke, 4, &parts[2]) && parts[0] <= kNoAllocScratchBytes &&
                      parts[1] <= kNoAllocScratchBytes && parts[2] <= kNoAllocScratchBytes;
    const size_t q_bytes = fits ? align256(parts[0]) : 0;
    const size_t key_bytes = fits ? align256(parts[1]) : 0;
    const size_t sel_bytes = fits ? align256(parts[2]) : 0;
    const size_t need = q_bytes + key_bytes + 2 * sel_bytes;
    if (!fits || need > kNoAllocScratchBytes)
      fail(ORDVEC_STATUS_BAD_ARGUMENT,
           "ovb_rankquant_search_noalloc: nq=" + std::to_string(nq) + ", n=" + std::to_string(ix.n) + ", k=" +
               std::to_string(ke) + " needs more than the " + std::to_string(kNoAllocScratchBytes) +
               " bytes (32 MiB) of scratch the allocation-free entry point has: use ovb_rankquant_search or "
               "smaller batches");
    uint8_t* base = scratch_base();
    float* qu = (float*)base;
    uint32_t* keys = (uint32_t*)(base + q_bytes);
    uint32_t* sel_keys = (uint32_t*)(base + q_bytes + key_bytes);
    uint32_t* sel_ids = (uint32_t*)(base + q_bytes + key_bytes + sel_bytes);
    cudaStream_t st = (cudaStream_t)stream;
    const double nbk = (double)(1u << ix.bits);
    const float inv_norm = 1.0f / (float)std::sqrt((double)ix.dim * ((nbk * nbk - 1.0) / 12.0));
    launch_l2_normalise(d_queries, nq, ix.dim, qu, st);
    launch_asym_scan(ix.codes.as<uint8_t>(), ix.n, ix.dim, ix.bits, qu, nq, inv_norm, keys, ix.n, st);
    SelectArgs a{keys, nullptr, nullptr, ix.n, ix.n, (uint32_t)ke, 32, bits_for(ix.n - 1), sel_keys, sel_ids};
    launch_select_rows(a, nq, nullptr, st);
    launch_keys_to_results(sel_keys, sel_ids, nq * ke, 0, 0, d_scores, d_ids, st);
  });
}
