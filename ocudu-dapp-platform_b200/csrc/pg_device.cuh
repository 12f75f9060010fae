// Device helpers shared by the pusch_b200 kernels.
#pragma once

#include <cstdint>

namespace pg {

// std::isnormal for device code: finite, non-zero and not subnormal.
__device__ __forceinline__ bool is_normal(float x)
{
  const float a = fabsf(x);
  return a >= 1.17549435e-38f && a <= 3.40282347e+38f;
}

// c(bit) .. c(bit + 31) of the TS 38.211 Section 5.2.1 Gold sequence with initialisation c_init
// (bit j of the result = c(bit + j)). tab holds 32 basis sequences of `words` words each, from
// position Nc = 1600: row 0 = x1 from (1, 0, ..., 0), row i + 1 = x2 from the unit state e_i; c is
// linear in c_init, so any sequence is x1 xor the rows of the set bits of c_init.
__device__ __forceinline__ uint32_t gold_word(const uint32_t* __restrict__ tab, uint32_t words, uint32_t c_init,
                                              uint32_t bit)
{
  const uint32_t w  = bit >> 5;
  const uint32_t sh = bit & 31u;
  uint32_t       lo = __ldg(tab + w), hi = __ldg(tab + w + 1);
#pragma unroll
  for (int i = 0; i < 31; ++i) {
    if ((c_init >> i) & 1u) {
      const uint32_t* b = tab + (size_t)(i + 1) * words;
      lo ^= __ldg(b + w);
      hi ^= __ldg(b + w + 1);
    }
  }
  return sh ? ((lo >> sh) | (hi << (32 - sh))) : lo;
}

} // namespace pg
