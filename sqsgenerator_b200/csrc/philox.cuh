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

PHILOX_HD uint32_t rotl32(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }

// xoshiro128** (Blackman and Vigna, "Scrambled linear pseudorandom number generators", ACM TOMS
// 2021): 128 bits of state, a 32-bit output per step (the starstar scrambler of the second word).
struct xoshiro128ss {
  uint32_t s0, s1, s2, s3;
  PHILOX_HD uint32_t next() {
    const uint32_t r = rotl32(s1 * 5u, 7) * 9u;
    const uint32_t t = s1 << 9;
    s2 ^= s0;
    s3 ^= s1;
    s1 ^= s2;
    s0 ^= s3;
    s2 ^= t;
    s3 = rotl32(s3, 11);
    return r;
  }
};

// The words of one configuration's shuffle of one part: a xoshiro128** generator whose state is one
// Philox4x32-10 block, counter (0, iteration, chain_lo, chain_hi << 8 | part) and key = seed, so that
// a configuration depends on (seed, id, part) alone; one block per configuration instead of one per
// four words. An all-zero block (the generator's one fixed point) becomes state (1, 0, 0, 0).
PHILOX_HD xoshiro128ss shuffle_words(uint32_t it, uint32_t c_lo, uint32_t c_hi, uint32_t k0, uint32_t k1) {
  const philox_ctr r = philox4x32_10(philox_ctr{0u, it, c_lo, c_hi}, k0, k1);
  xoshiro128ss g{r.x, r.y, r.z, r.w};
  if ((r.x | r.y | r.z | r.w) == 0u) g.s0 = 1u;
  return g;
}

}  // namespace sqsg
