// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies with the published multipliers
// and Weyl key increments. Host and device.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define PHILOX_HD __host__ __device__ __forceinline__
#else
#define PHILOX_HD inline
#endif

namespace sqsg {

struct philox_ctr {
  uint32_t x, y, z, w;
};

PHILOX_HD uint32_t mulhilo32(uint32_t a, uint32_t b, uint32_t* hi) {
  uint64_t p = static_cast<uint64_t>(a) * b;
  *hi = static_cast<uint32_t>(p >> 32);
  return static_cast<uint32_t>(p);
}

PHILOX_HD philox_ctr philox4x32_10(philox_ctr c, uint32_t k0, uint32_t k1) {
  constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, hi1;
    uint32_t lo0 = mulhilo32(M0, c.x, &hi0);
    uint32_t lo1 = mulhilo32(M1, c.z, &hi1);
    c = philox_ctr{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += W0;
    k1 += W1;
  }
  return c;
}

}  // namespace sqsg
