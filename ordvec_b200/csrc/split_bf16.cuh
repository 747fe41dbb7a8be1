// Exact BF16 expansion of packed RankQuant codes for the split-BF16 tensor-core
// kernels: each centred code (code - c), c = (2^B - 1) / 2, has at most 4
// significant bits, so its bf16 is exact.  A 16-entry nibble table lives in
// the lanes of a warp (lanes 16..31 repeat 0..15) and is read with warp
// shuffles: one shuffle per 4-bit group of MSB-first codes gives their bf16
// pair (b=2), two pairs (b=1, two tables) or one value (b=4).
#pragma once
#include <stdint.h>

namespace ovb {
namespace tc {

// upper 16 bits of an f32 = its bf16 when the low 16 bits are zero (exact here)
__device__ __forceinline__ uint32_t bf16_bits(float x) { return __float_as_uint(x) >> 16; }

// The lane's entry of the 16-entry nibble table (lanes 16..31 repeat 0..15).
template <int BITS>
__device__ __forceinline__ void nibble_table(uint32_t lane, uint32_t& t0, uint32_t& t1) {
  const uint32_t v = lane & 15;
  if (BITS == 2) {  // two codes: c0 = v >> 2 (first), c1 = v & 3
    t0 = bf16_bits((float)(v >> 2) - 1.5f) | (bf16_bits((float)(v & 3) - 1.5f) << 16);
    t1 = 0;
  } else if (BITS == 1) {  // four codes, first in bit 3
    t0 = bf16_bits((float)((v >> 3) & 1) - 0.5f) | (bf16_bits((float)((v >> 2) & 1) - 0.5f) << 16);
    t1 = bf16_bits((float)((v >> 1) & 1) - 0.5f) | (bf16_bits((float)(v & 1) - 0.5f) << 16);
  } else {  // one code
    t0 = bf16_bits((float)v - 7.5f);
    t1 = 0;
  }
}

// nibble k (0..7) of a little-endian word of MSB-first bytes: byte k/2, high
// half first
__device__ __forceinline__ uint32_t nib(uint32_t w, int k) { return (w >> (8 * (k >> 1) + ((k & 1) ? 0 : 4))) & 15; }

}  // namespace tc
}  // namespace ovb
