// Counter-based uniforms shared by the samplers: one double per (seed, item, position),
// so a sample does not depend on how items are grouped into tiles or launches.
#pragma once
#include <cuda_runtime.h>

namespace rgs {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2,
// 3", SC 2011): counter (item, position, stream, 0), key = seed.
__device__ __forceinline__ uint4 philox4x32_10(uint4 ctr, uint2 key) {
  const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    const unsigned hi0 = __umulhi(M0, ctr.x), lo0 = M0 * ctr.x;
    const unsigned hi1 = __umulhi(M1, ctr.z), lo1 = M1 * ctr.z;
    ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
    key.x += W0;
    key.y += W1;
  }
  return ctr;
}

// Uniform double in [0, 1) with 53 random bits.
__device__ __forceinline__ double philox_uniform(unsigned long long seed, unsigned long long item, int position) {
  const uint4 r = philox4x32_10(make_uint4((unsigned)item, (unsigned)(item >> 32), (unsigned)position, 0u),
                                make_uint2((unsigned)seed, (unsigned)(seed >> 32)));
  const unsigned long long bits = (((unsigned long long)r.x << 32) | r.y) >> 11;
  return (double)bits * 0x1.0p-53;
}

}  // namespace rgs
