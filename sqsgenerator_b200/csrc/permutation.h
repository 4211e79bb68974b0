// Multiset permutation arithmetic on u64 ranks with 128-bit intermediates, usable on host and device.
//
// Restates include/sqsgen/core/permutation.h:17-102 of the reference. Ranks there are boost::cpp_int;
// the reference parser refuses jobs whose permutation count exceeds u64
// (include/sqsgen/io/config/combined.h:88-95), so every rank it iterates fits in u64. Products such as
// total * hist[j] stay below 2^96 because counts are below 2^32.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define SQSG_HD __host__ __device__ __forceinline__
#else
#define SQSG_HD inline
#endif

namespace sqsg {

struct u96 {
  uint64_t lo;
  uint32_t hi;
};

// a * b for a < 2^64, b < 2^32.
SQSG_HD u96 mul_64x32(uint64_t a, uint32_t b) {
  uint64_t lo = (a & 0xffffffffull) * b;
  uint64_t mid = (a >> 32) * b;
  uint64_t r_lo = lo + (mid << 32);
  uint32_t carry = r_lo < lo ? 1u : 0u;
  return u96{r_lo, static_cast<uint32_t>(mid >> 32) + carry};
}

// x / d for d > 0; *overflow is set when the quotient does not fit 64 bits.
SQSG_HD uint64_t div_96x32(u96 x, uint32_t d, bool* overflow) {
  uint64_t r = 0;
  uint32_t limbs[3] = {static_cast<uint32_t>(x.lo), static_cast<uint32_t>(x.lo >> 32), x.hi};
  uint32_t q[3];
  for (int k = 2; k >= 0; --k) {
    uint64_t cur = (r << 32) | limbs[k];
    q[k] = static_cast<uint32_t>(cur / d);
    r = cur % d;
  }
  if (q[2] != 0 && overflow) *overflow = true;
  return (static_cast<uint64_t>(q[1]) << 32) | q[0];
}

// core/permutation.h:17-32 — number of distinct arrangements of a multiset with the given counts,
// as a product of binomials; returns false on u64 overflow.
SQSG_HD bool num_permutations_counts(const uint32_t* counts, int k, uint64_t* out) {
  uint64_t total = 1;
  uint32_t m = 0;
  for (int s = 0; s < k; ++s) {
    uint64_t binom = 1;
    for (uint32_t t = 1; t <= counts[s]; ++t) {
      bool of = false;
      binom = div_96x32(mul_64x32(binom, m + t), t, &of);
      if (of) return false;
    }
    m += counts[s];
    // total * binom may exceed 96 bits; check with a division.
    if (binom != 0 && total > UINT64_MAX / binom) return false;
    total *= binom;
  }
  *out = total;
  return true;
}

// core/permutation.h:34-50 — 1-based rank of a configuration with dense values 0..k-1 (k <= 256).
// hist is caller scratch of k entries.
SQSG_HD uint64_t rank_permutation(const uint8_t* conf, uint32_t n, uint32_t* hist, int k) {
  for (int j = 0; j < k; ++j) hist[j] = 0;
  uint64_t rank = 1, suffix = 1;
  for (uint32_t i = 0; i < n; i++) {
    uint32_t x = conf[(n - 1) - i];
    hist[x]++;
    for (uint32_t j = 0; j < x; j++) rank += div_96x32(mul_64x32(suffix, hist[j]), hist[x], nullptr);
    suffix = div_96x32(mul_64x32(suffix, i + 1), hist[x], nullptr);
  }
  return rank;
}

}  // namespace sqsg
