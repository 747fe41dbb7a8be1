// Self-test of the tensor-core kernels' bounded waits: one thread waits on an
// mbarrier that nothing arrives at, through the same bounded wait the scan
// kernels use, and reports whether the wait gave up and after how long.  The
// wait ends by its own limit (about one second), so the test exercises the
// timeout path without a fault or a hang, and the context stays usable.
#include "ovb_kernels.h"
#include "tc_common.cuh"

namespace ovb {

namespace {

__global__ void wait_probe_kernel(uint32_t* __restrict__ out) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) tc::mbar_init(&bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint64_t t0 = tc::global_ns();
    const bool completed = tc::mbar_wait(&bar, 0);  // phase 0 never completes: no arrive is issued
    const uint64_t dt = tc::global_ns() - t0;
    out[0] = completed ? 0u : 1u;
    out[1] = (uint32_t)dt;
    out[2] = (uint32_t)(dt >> 32);
  }
}

}  // namespace

void launch_wait_probe(uint32_t* d_out, cudaStream_t stream) {
  wait_probe_kernel<<<1, 32, 0, stream>>>(d_out);
  launched();
}

}  // namespace ovb
