// Shared device/host helpers for the ordvec B200 scan kernels.
//
// Ordering convention used by every kernel: a candidate is a 64-bit logical
// key  (key32 << 32) | id32  and SMALLER IS BETTER.  key32 is a monotone
// encoding of the score in the direction the reference ranks it:
//   * sign hamming (src/sign_bitmap.rs:216-222, ascending)   -> key32 = hamming
//   * bitmap overlap (src/bitmap.rs:274-285, descending)     -> key32 = n_top - overlap
//   * float scores (src/util.rs:375-385, total_cmp desc)      -> key32 = desc_key(score)
// and id32 is the global row id, so ties break by ascending id exactly as the
// reference's TopK / select_nth composite keys do.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>

namespace ovb {

#define OVB_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      throw ::ovb::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

// Lets `kernel` take as much dynamic shared memory as the current device allows
// beside its static shared memory, once per (kernel, device).  A launch needs
// the opt-in once static + dynamic exceed 48 KiB; setting the limit to the
// launch's own size instead would let two host threads with different sizes
// lower it under each other's launches.
template <class K>
void allow_dynamic_smem(K* kernel) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  OVB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({(const void*)kernel, dev})) return;
  int optin = 0;
  OVB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  OVB_CUDA(cudaFuncGetAttributes(&fa, (const void*)kernel));
  OVB_CUDA(cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                optin - (int)fa.sharedSizeBytes));
  done.insert({(const void*)kernel, dev});
}

// Kernel launches issued by this thread (benchmark instrumentation).  A launch
// error names the launching function and line.
extern thread_local uint64_t tl_launch_counter;
inline void launched(const char* fn = __builtin_FUNCTION(), int line = __builtin_LINE()) {
  tl_launch_counter++;
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    throw CudaError(std::string("kernel launch in ") + fn + " (line " + std::to_string(line) + "): " +
                    cudaGetErrorString(e));
}

// f32::total_cmp ascending maps to unsigned ascending of
// bits ^ (sign ? 0xFFFFFFFF : 0x80000000); descending score -> complement.
__host__ __device__ __forceinline__ uint32_t asc_key(float f) {
#ifdef __CUDA_ARCH__
  uint32_t b = __float_as_uint(f);
#else
  uint32_t b;
  memcpy(&b, &f, 4);
#endif
  return b ^ ((b >> 31) ? 0xFFFFFFFFu : 0x80000000u);
}
__host__ __device__ __forceinline__ uint32_t desc_key(float f) { return ~asc_key(f); }
__host__ __device__ __forceinline__ float desc_key_to_float(uint32_t k) {
  uint32_t a = ~k;
  uint32_t b = (a >> 31) ? (a ^ 0x80000000u) : ~a;
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float f;
  memcpy(&f, &b, 4);
  return f;
#endif
}

constexpr uint32_t kSentinelKey = 0xFFFFFFFFu;
constexpr uint32_t kSentinelId = 0xFFFFFFFFu;

__host__ __device__ __forceinline__ uint32_t bits_for(uint64_t max_value) {
  uint32_t b = 0;
  while (b < 64 && (max_value >> b) != 0) b++;
  return b;
}

inline unsigned ceil_div(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace ovb
