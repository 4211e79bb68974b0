// Device side of the SQS engine (included by the kernel translation units kernel_*.cu).
//
// Per configuration a thread
//   1. (random mode) Fisher-Yates-shuffles every window of every part of the packed initial
//      arrangement with the words of a xoshiro128** generator seeded by one Philox4x32-10 block
//      (key = seed, counter = (0, 0, configuration id, part); philox.cuh) and the reference's bounded
//      draw p = (x * i) >> 32 (include/sqsgen/core/shuffle.h:28-50); a window of two species draws
//      its rarer species' sites by Floyd's sampling instead (same distribution, fewer draws);
//   2. counts ordered bonds (s, species[i], species[j]) over the part's pairs (optimization.h:74-77);
//   3. evaluates the objective in T with the reference's loop order and no FMA contraction
//      (optimization.h:79-103), summing parts left to right from T(0) (sqs.h:417-418, fold.h:51-53);
//   4. takes part in the warp's best-N bookkeeping (results.h:42-99, sqs.h:421-438);
//   5. (systematic mode) steps to the lexicographically next multiset permutation
//      (permutation.h:80-102) inside the window.
#pragma once

#include <cfloat>
#include <cstdint>
#include <cstring>

#include "engine.cuh"
#include "permutation.h"
#include "philox.cuh"

namespace sqsg {

template <class T> struct FP;
template <> struct FP<double> {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double cvt(uint32_t n) { return __uint2double_rn(n); }
  static __device__ __forceinline__ double maxv() { return DBL_MAX; }
};
template <> struct FP<float> {
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float cvt(uint32_t n) { return __uint2float_rn(n); }
  static __device__ __forceinline__ float maxv() { return FLT_MAX; }
};


// Byte offset of site x inside a lane's species column: words of four sites are interleaved across
// the kBlock lanes, so both a uniform site (bond counting) and per-lane random sites (shuffling) hit
// distinct banks.
__device__ __forceinline__ uint32_t site_off(uint32_t x) { return (x >> 2) * (kBlock * 4) + (x & 3); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ------------------------------------------------------------------------------ bulk-copy staging
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Non-multicast 1D bulk copy global -> this CTA's shared memory (TMA unit), completing on bar.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for the phase `parity` of bar, bounded by limit_ns of the global timer (read every 64 polls);
// false when the bound ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long limit_ns) {
  const uint32_t addr = smem_u32(bar);
  const unsigned long long t0 = global_ns();
  for (uint32_t it = 1;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 63u) == 0 && global_ns() - t0 > limit_ns) return false;
  }
}

// ------------------------------------------------------------------------------ per-part kernels
__device__ __forceinline__ uint8_t* part_base(uint8_t* smem, const PartDesc& P) { return smem + P.smem_off; }

__device__ __forceinline__ void init_column(uint8_t* smem, const PartDesc& P, int t) {
  const uint32_t* sp = reinterpret_cast<const uint32_t*>(part_base(smem, P) + P.species_off);
  uint32_t* col = reinterpret_cast<uint32_t*>(part_base(smem, P) + P.col_off) + t;
  const uint32_t words = (P.n_sites + 3) >> 2;
  for (uint32_t w = 0; w < words; ++w) col[w * kBlock] = sp[w];
}

// Ordered bond counts of the lane's configuration into its histogram (16-bit fields).
// Stream word k: from the job blob through the read-only L1 path (GLOBAL; every lane of a warp reads
// the same address, one request, and the stream stays L1-resident for all CTAs of the SM) or from
// the staged copy in shared memory.
template <bool GLOBAL> __device__ __forceinline__ uint32_t stream_word(const uint32_t* st, uint32_t k) {
  if (GLOBAL) return __ldg(st + k);
  return st[k];
}

template <int KW, bool GLOBAL>
__device__ __forceinline__ void count_part_from(uint8_t* smem, const uint32_t* __restrict__ st, const PartDesc& P,
                                                int t) {
  uint8_t* part = part_base(smem, P);
  const uint8_t* col = part + P.col_off + 4 * t;
  uint32_t* hist = reinterpret_cast<uint32_t*>(part + P.hist_off) + t;
  const uint32_t K = P.n_species, hw = P.hw, words = P.stream_words;
  const uint32_t nh = P.n_shells * K * hw;
  for (uint32_t w = 0; w < nh; ++w) hist[w * kBlock] = 0;
  uint32_t pos = 0;
  if (P.stream_narrow) {
    // one header word per group, then two 16-bit column offsets per word
    while (pos < words) {
      const uint32_t hdr = stream_word<GLOBAL>(st, pos);
      const uint32_t s = (hdr >> 16) & 0xffu, cnt = hdr >> 24;
      const uint32_t ci = col[hdr & 0xffffu] >> 3;
      const uint32_t* js = st + pos + 1;
      const uint32_t pairs = cnt >> 1;
      uint32_t* h = hist + ((s * K + ci) * hw) * kBlock;
      if (KW == 1) {
        uint32_t row = 0;
#pragma unroll 4
        for (uint32_t e = 0; e < pairs; ++e) {
          const uint32_t w2 = stream_word<GLOBAL>(js, e);
          row += (1u << col[w2 & 0xffffu]) + (1u << col[w2 >> 16]);
        }
        if (cnt & 1u) row += 1u << col[stream_word<GLOBAL>(js, pairs) & 0xffffu];
        h[0] += __byte_perm(row, 0, 0x4140);
        if (hw > 1) h[kBlock] += __byte_perm(row, 0, 0x4342);
      } else {
        unsigned long long row = 0;
#pragma unroll 4
        for (uint32_t e = 0; e < pairs; ++e) {
          const uint32_t w2 = stream_word<GLOBAL>(js, e);
          row += (1ull << col[w2 & 0xffffu]) + (1ull << col[w2 >> 16]);
        }
        if (cnt & 1u) row += 1ull << col[stream_word<GLOBAL>(js, pairs) & 0xffffu];
        const uint32_t lo = static_cast<uint32_t>(row), hi = static_cast<uint32_t>(row >> 32);
        h[0] += __byte_perm(lo, 0, 0x4140);
        if (hw > 1) h[kBlock] += __byte_perm(lo, 0, 0x4342);
        if (hw > 2) h[2 * kBlock] += __byte_perm(hi, 0, 0x4140);
        if (hw > 3) h[3 * kBlock] += __byte_perm(hi, 0, 0x4342);
      }
      pos += 1 + ((cnt + 1) >> 1);
    }
    return;
  }
  while (pos < words) {
    const uint32_t hdr = stream_word<GLOBAL>(st, pos);
    const uint32_t ioff = stream_word<GLOBAL>(st, pos + 1);
    const uint32_t s = hdr & 0xffu, cnt = (hdr >> 8) & 0xffu;
    const uint32_t ci = col[ioff] >> 3;
    const uint32_t* js = st + pos + 2;
    uint32_t* h = hist + ((s * K + ci) * hw) * kBlock;
    if (KW == 1) {
      uint32_t row = 0;
#pragma unroll 4
      for (uint32_t e = 0; e < cnt; ++e) row += 1u << col[stream_word<GLOBAL>(js, e)];
      h[0] += __byte_perm(row, 0, 0x4140);
      if (hw > 1) h[kBlock] += __byte_perm(row, 0, 0x4342);
    } else {
      unsigned long long row = 0;
#pragma unroll 4
      for (uint32_t e = 0; e < cnt; ++e) row += 1ull << col[stream_word<GLOBAL>(js, e)];
      const uint32_t lo = static_cast<uint32_t>(row), hi = static_cast<uint32_t>(row >> 32);
      h[0] += __byte_perm(lo, 0, 0x4140);
      if (hw > 1) h[kBlock] += __byte_perm(lo, 0, 0x4342);
      if (hw > 2) h[2 * kBlock] += __byte_perm(hi, 0, 0x4140);
      if (hw > 3) h[3 * kBlock] += __byte_perm(hi, 0, 0x4342);
    }
    pos += 2 + cnt;
  }
}

template <int KW>
__device__ __forceinline__ void count_part(uint8_t* smem, const uint8_t* blob, const PartDesc& P, int t) {
  if (P.stream_global)
    count_part_from<KW, true>(smem, reinterpret_cast<const uint32_t*>(blob + P.blob_off + P.stream_off), P, t);
  else
    count_part_from<KW, false>(smem, reinterpret_cast<const uint32_t*>(part_base(smem, P) + P.stream_off), P, t);
}

__device__ __forceinline__ uint32_t bond(const uint32_t* hist, uint32_t K, uint32_t hw, uint32_t s, uint32_t a,
                                         uint32_t b) {
  return (hist[((s * K + a) * hw + (b >> 1)) * kBlock] >> ((b & 1u) * 16u)) & 0xffffu;
}

// core/optimization.h:79-103 on the lane's histogram. With `sro` non-null the SRO cube is written
// row-major (the reference's sro tensor, symmetric in the species indices).
template <class T>
__device__ __forceinline__ T objective_part(uint8_t* smem, const PartDesc& P, int t, T* sro = nullptr) {
  using F = FP<T>;
  const uint8_t* part = part_base(smem, P);
  const uint32_t* hist = reinterpret_cast<const uint32_t*>(part + P.hist_off) + t;
  const uint32_t S = P.n_shells, K = P.n_species, hw = P.hw, skk = S * K * K;
  const T* f = reinterpret_cast<const T*>(part + P.cube_off);
  const T* w = f + skk;
  const T* tg = w + skk;
  T obj = T(0);
  for (uint32_t s = 0; s < S; ++s)
    for (uint32_t xi = 0; xi < K; ++xi) {
      const uint32_t d = (s * K + xi) * K + xi;
      const T sig = F::sub(T(1), F::mul(F::cvt(bond(hist, K, hw, s, xi, xi)), f[d]));
      if (sro) sro[d] = sig;
      T diff = F::sub(sig, tg[d]);
      diff = diff > T(0) ? diff : -diff;
      obj = F::add(obj, F::mul(w[d], diff));
      for (uint32_t eta = xi + 1; eta < K; ++eta) {
        const uint32_t u = (s * K + xi) * K + eta;
        const uint32_t nb = bond(hist, K, hw, s, xi, eta) + bond(hist, K, hw, s, eta, xi);
        const T sg = F::sub(T(1), F::mul(F::cvt(nb), f[u]));
        if (sro) {
          sro[u] = sg;
          sro[(s * K + eta) * K + xi] = sg;
        }
        T df = F::sub(sg, tg[u]);
        df = df > T(0) ? df : -df;
        obj = F::add(obj, F::mul(w[u], df));
      }
    }
  return obj;
}

__device__ __forceinline__ void swap_draw(uint8_t* col, uint32_t lo, uint32_t i, uint32_t x) {
  const uint32_t p = __umulhi(x, i);  // (x * i) >> 32, core/shuffle.h:28-32 on a 32-bit word
  const uint32_t a = site_off(lo + i - 1), b = site_off(lo + p);
  const uint8_t va = col[a], vb = col[b];
  col[a] = vb;
  col[b] = va;
}

// Floyd's sampling of an m-subset of a window of n sites (Bentley and Floyd, "A sample of brilliance",
// CACM 30(9), 1987): for j = n-m .. n-1 draw t uniform in [0, j] and take t, or j when t is taken. The
// window starts filled with the other species, so "taken" is "holds the rarer species". Every
// m-subset is equally likely, which is the distribution of the window's sites of that species after
// a Fisher-Yates shuffle, with m draws instead of n - 1.
__device__ __forceinline__ void floyd_window(uint8_t* col, uint32_t lo, uint32_t n, uint32_t word,
                                             xoshiro128ss& words) {
  const uint32_t m = word & 0xffffu;
  const uint8_t rare = static_cast<uint8_t>(word >> 16);
  for (uint32_t j = n - m; j < n; ++j) {
    const uint32_t at = site_off(lo + __umulhi(words.next(), j + 1));  // (x * (j+1)) >> 32: t in [0, j]
    col[col[at] == rare ? site_off(lo + j) : at] = rare;
  }
}

// core/shuffle.h:39-50 with the words of shuffle_words (philox.cuh): a xoshiro128** generator seeded
// by the Philox4x32-10 block of (seed; iteration, chain, part); the windows draw one after another. A
// window of exactly two species (draw word != 0, staged after the window bounds) takes Floyd's
// sampling of its rarer species' sites instead of the swaps; the staged initial arrangement holds the
// other species on it.
__device__ __forceinline__ void shuffle_part(uint8_t* smem, const PartDesc& P, int t, uint32_t it,
                                             unsigned long long chain, uint32_t part, uint32_t k0, uint32_t k1) {
  uint8_t* col = part_base(smem, P) + P.col_off + 4 * t;
  const uint32_t* win = reinterpret_cast<const uint32_t*>(part_base(smem, P) + P.win_off);
  xoshiro128ss words =
      shuffle_words(it, static_cast<uint32_t>(chain), (static_cast<uint32_t>(chain >> 32) << 8) | part, k0, k1);
  for (uint32_t wi = 0; wi < P.n_windows; ++wi) {
    const uint32_t lo = win[2 * wi], n = win[2 * wi + 1] - lo, fw = win[2 * P.n_windows + wi];
    if (fw) {
      floyd_window(col, lo, n, fw, words);
    } else {
      for (uint32_t i = n; i > 1; --i) swap_draw(col, lo, i, words.next());
    }
  }
}

// ------------------------------------------------------------------------------ reference random stream
// Debug mode that reproduces the reference's seeded single-thread trajectories. Its random words are
// rapidrand's (core/shuffle.h:23-26): the state advances by rapidhash's secret 0 per draw and the
// word is rapidhash's mix of (state, state ^ secret 1), the 64x64->128-bit product folded by xor
// (core/helpers/rapidhash.h:129-131,149-213); the shuffle uses its low 32 bits (core/shuffle.h:28-32).
constexpr unsigned long long kRapidSecret0 = 0x2d358dccaa6c78a5ull;
constexpr unsigned long long kRapidSecret1 = 0x8bb84b93962eacc9ull;

__device__ __forceinline__ uint32_t rapid_next(unsigned long long& s) {
  s += kRapidSecret0;
  const unsigned long long b = s ^ kRapidSecret1;
  return static_cast<uint32_t>((s * b) ^ __umul64hi(s, b));
}

// core/shuffle.h:39-50 on the reference's stream: Fisher-Yates per window, one word per step.
__device__ __forceinline__ void shuffle_part_rapid(uint8_t* smem, const PartDesc& P, int t, unsigned long long& s) {
  uint8_t* col = part_base(smem, P) + P.col_off + 4 * t;
  const uint32_t* win = reinterpret_cast<const uint32_t*>(part_base(smem, P) + P.win_off);
  for (uint32_t wi = 0; wi < P.n_windows; ++wi) {
    const uint32_t lo = win[2 * wi];
    for (uint32_t i = win[2 * wi + 1] - lo; i > 1; --i) swap_draw(col, lo, i, rapid_next(s));
  }
}

// The reference's thread-pool blocks over [0, total) (sqs.h:461-466): chain_rem blocks of
// chain_block + 1 configurations, then blocks of chain_block; the last block ends at total.
__device__ __forceinline__ uint64_t chain_block_start(const JobDesc& J, uint64_t b) {
  return b * J.chain_block + (b < J.chain_rem ? b : J.chain_rem);
}
__device__ __forceinline__ uint64_t chain_block_end(const JobDesc& J, uint64_t b) {
  return b + 1 == J.chain_blocks ? J.total : chain_block_start(J, b + 1);
}
__device__ __forceinline__ uint64_t chain_block_of(const JobDesc& J, uint64_t id) {
  const uint64_t edge = J.chain_rem * (J.chain_block + 1);
  const uint64_t b = id < edge ? id / (J.chain_block + 1) : J.chain_rem + (id - edge) / J.chain_block;
  return b < J.chain_blocks ? b : J.chain_blocks - 1;
}
// Stream state of a part at the start of the block that begins with configuration `first`: a single
// thread runs the blocks in order, each configuration shuffles once, each shuffle draws chain_draws.
__device__ __forceinline__ unsigned long long chain_state(const JobDesc& J, const PartDesc& P, uint64_t first) {
  return J.seed + first * static_cast<unsigned long long>(P.chain_draws) * kRapidSecret0;
}

// core/permutation.h:80-102 on the lane's window bytes.
__device__ __forceinline__ void next_permutation(uint8_t* col, uint32_t lo, uint32_t n) {
  if (n < 2) return;
  int k = static_cast<int>(n) - 2;
  uint8_t right = col[site_off(lo + n - 1)];
  uint8_t ak = col[site_off(lo + k)];
  while (ak >= right) {
    if (--k < 0) return;
    right = ak;
    ak = col[site_off(lo + k)];
  }
  int l = static_cast<int>(n) - 1;
  uint8_t al = col[site_off(lo + l)];
  while (ak >= al) al = col[site_off(lo + --l)];
  col[site_off(lo + k)] = al;
  col[site_off(lo + l)] = ak;
  for (int a = k + 1, b = static_cast<int>(n) - 1; a < b; ++a, --b) {
    const uint32_t oa = site_off(lo + a), ob = site_off(lo + b);
    const uint8_t va = col[oa];
    col[oa] = col[ob];
    col[ob] = va;
  }
}

// core/permutation.h:52-78 inside the window with the dense remap of core/shuffle.h:73-87.
__device__ __forceinline__ void unrank_window(uint8_t* col, const PartDesc& P, uint32_t lo, uint32_t n,
                                              uint64_t rank, uint64_t total) {
  uint32_t h[kMaxSpecies];
  const uint32_t k = P.unrank_k;
  for (uint32_t j = 0; j < kMaxSpecies; ++j) h[j] = P.unrank_hist[j];
  for (uint32_t i = 0; i < n; ++i) {
    for (uint32_t j = 0; j < k; ++j) {
      const uint64_t suffix = div_96x32(mul_64x32(total, h[j]), n - i, nullptr);
      if (rank <= suffix) {
        col[site_off(lo + i)] = static_cast<uint8_t>(P.unrank_rev[j] << 3);
        total = suffix;
        h[j]--;
        break;
      }
      rank -= suffix;
    }
  }
}

// ------------------------------------------------------------------------------ objective levels
__device__ __forceinline__ uint32_t level_hash(unsigned long long key, uint32_t mask) {
  return static_cast<uint32_t>(mix64(key)) & mask;
}

// Keys above the job's threshold can never be among the final keep+1 levels and are dropped. A probe
// sequence is bounded; a key that finds no slot marks the table inexact (the host then rebuilds the
// levels from the records), and from then on the table takes no more keys.
constexpr int kLevelProbes = 64;

__device__ __forceinline__ void global_level_add(const JobDesc& J, unsigned long long key, unsigned long long count,
                                                 unsigned int sa, unsigned int sb) {
  if (key > *reinterpret_cast<volatile unsigned long long*>(&J.counters[kThreshold])) return;
  if (*reinterpret_cast<volatile unsigned long long*>(&J.counters[kLevelOverflow]) != 0ull) return;
  uint32_t h = level_hash(key, kLevelSlots - 1);
  for (int probe = 0; probe < kLevelProbes; ++probe, h = (h + 1) & (kLevelSlots - 1)) {
    LevelSlot& slot = J.levels[h];
    const unsigned long long prev = atomicCAS(&slot.key, 0ull, key);
    if (prev == 0ull || prev == key) {
      atomicAdd(&slot.count, count);
      atomicAdd(&slot.sum_a, sa);
      atomicAdd(&slot.sum_b, sb);
      return;
    }
  }
  atomicAdd(&J.counters[kLevelOverflow], 1ull);
}

__device__ __forceinline__ void cta_level_add(LevelSlot* tab, const JobDesc& J, unsigned long long key,
                                              unsigned long long count, unsigned int sa, unsigned int sb) {
  uint32_t h = level_hash(key, kCtaLevelSlots - 1);
  for (int probe = 0; probe < kCtaLevelSlots; ++probe, h = (h + 1) & (kCtaLevelSlots - 1)) {
    const unsigned long long prev = atomicCAS(&tab[h].key, 0ull, key);
    if (prev == 0ull || prev == key) {
      atomicAdd(&tab[h].count, count);
      atomicAdd(&tab[h].sum_a, sa);
      atomicAdd(&tab[h].sum_b, sb);
      return;
    }
  }
  global_level_add(J, key, count, sa, sb);
}

// Moves the CTA's level entries that are still at or below the job's threshold into the job table.
__device__ __forceinline__ void flush_levels(LevelSlot* tab, const JobDesc& J) {
  for (int i = threadIdx.x; i < kCtaLevelSlots; i += kBlock) {
    LevelSlot& slot = tab[i];
    if (slot.key) {
      global_level_add(J, slot.key, slot.count, slot.sum_a, slot.sum_b);
      slot.key = 0;
      slot.count = 0;
      slot.sum_a = 0;
      slot.sum_b = 0;
    }
  }
}

// ------------------------------------------------------------------------------ best-N bookkeeping
// Each warp keeps the best distinct objectives it has seen, ascending: with keep <= 31 one entry per
// lane (32 entries in registers), with larger keep a list of big_len >= keep+1 entries in shared
// memory. Its (keep+1)-th entry bounds the job's (keep+1)-th best distinct objective from above, like
// the reference's search threshold nth_best(keep) (results.h:78-82, sqs.h:203-206); the minimum over
// warps is kept in the job's threshold counter. Every configuration whose objective is at or below
// the current bound is appended to the candidate buffer, so the buffer holds every configuration at
// or below the final (keep+1)-th best distinct objective.
struct WarpState {
  double list;          // lane's entry of the register list (+inf = empty); unused with `big`
  double list_thr;      // warp-uniform (keep+1)-th entry
  double* big;          // keep >= 32: this warp's list in shared memory (nullptr otherwise)
  uint32_t big_len;
  unsigned long long published_thr, published_best;
  bool records_full;    // lane 0: the job's record buffer is known to be full (it never empties)
  // Called by every thread of the warp at a job switch.
  __device__ void reset(const JobDesc& J, uint8_t* smem) {
    list = __longlong_as_double(0x7ff0000000000000ll);
    list_thr = list;
    published_thr = ~0ull;
    published_best = ~0ull;
    records_full = false;
    big = nullptr;
    big_len = J.big_len;
    if (big_len) {
      big = reinterpret_cast<double*>(smem + J.big_off) + (threadIdx.x >> 5) * big_len;
      for (uint32_t k = threadIdx.x & 31; k < big_len; k += 32) big[k] = list;
      __syncwarp();
    }
  }
};

struct BigUpdate {
  double thr;
  bool moved;
};

// The shared-memory list (keep >= 32): membership of each lane's value by binary search, then one
// insertion per distinct new value below the (keep+1)-th entry, lane order; an insertion at `pos`
// moves entries [pos, len-1) up by one, highest block of 32 first (each block is read before it is
// written, and its lowest entry reads the block below, which is written later). Rare after the first
// tiles, so it is kept out of line.
static __device__ __noinline__ BigUpdate big_list_update(double* L, uint32_t n, double v_mine, bool fresh, uint32_t keep,
                                                  double thr) {
  const int lane = threadIdx.x & 31;
  if (fresh) {
    uint32_t lo = 0, hi = n;  // first entry >= v_mine
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (L[mid] < v_mine)
        lo = mid + 1;
      else
        hi = mid;
    }
    if (lo < n && L[lo] == v_mine) fresh = false;
  }
  unsigned fm = __ballot_sync(0xffffffffu, fresh);
  const bool moved = fm != 0;
  while (fm) {
    const double v = __shfl_sync(0xffffffffu, v_mine, __ffs(fm) - 1);
    fm &= ~__ballot_sync(0xffffffffu, v_mine == v);  // lanes with the same value: one insertion
    if (v < thr) {
      uint32_t c = 0;
      for (uint32_t k = lane; k < n; k += 32) c += L[k] < v ? 1u : 0u;
      const uint32_t pos = __reduce_add_sync(0xffffffffu, c);
      for (int blk = static_cast<int>(n >> 5) - 1; blk >= static_cast<int>(pos >> 5); --blk) {
        const uint32_t idx = static_cast<uint32_t>(blk) * 32 + lane;
        const double nv = idx > pos ? L[idx - 1] : v;
        __syncwarp();
        if (idx >= pos) L[idx] = nv;
        __syncwarp();
      }
      thr = L[keep];
    }
  }
  return BigUpdate{thr, moved};
}

// Per-warp level accumulators of the bit-mask path, indexed by position in the warp list: count,
// low and high checksum halves of the configurations kept at list[i] (3 x 32 words per warp). While
// the list does not change, a kept value is at the position its lower-bound search found, so each
// lane adds itself there with three shared-memory atomics instead of the warp looping over distinct
// values; before the list changes and at the end of every tile the warp moves them into the CTA table.
// (Register list only: with a shared-memory list the per-value loop runs instead.)
static __shared__ uint32_t s_wacc[kBlock / 32 * 96];

__device__ __forceinline__ uint32_t* warp_acc() { return s_wacc + (threadIdx.x >> 5) * 96; }

__device__ __forceinline__ void warp_acc_flush(const WarpState& ws, LevelSlot* ctab, const JobDesc& J) {
  __syncwarp();
  uint32_t* acc = warp_acc();
  const int lane = threadIdx.x & 31;
  const uint32_t c = acc[lane];
  if (c) {
    cta_level_add(ctab, J, ord_bits(ws.list), c, acc[32 + lane], acc[64 + lane]);
    acc[lane] = 0;
    acc[32 + lane] = 0;
    acc[64 + lane] = 0;
  }
  __syncwarp();
}

template <class T>
__device__ __forceinline__ void write_trace(const JobDesc& J, uint8_t* smem, uint64_t g, T total, uint64_t id,
                                            int t) {
  if (g >= J.trace_capacity) return;
  uint8_t* sp = J.trace_species + g * J.trace_species_stride;
  uint32_t* bd = J.trace_bonds + g * J.trace_bonds_stride;
  for (uint32_t p = 0; p < J.n_parts; ++p) {
    const PartDesc& P = J.parts[p];
    const uint8_t* part = part_base(smem, P);
    const uint8_t* col = part + P.col_off + 4 * t;
    const uint32_t* hist = reinterpret_cast<const uint32_t*>(part + P.hist_off) + t;
    for (uint32_t x = 0; x < P.n_sites; ++x) sp[P.trace_species_off + x] = col[site_off(x)] >> 3;
    const uint32_t S = P.n_shells, K = P.n_species;
    for (uint32_t s = 0; s < S; ++s)
      for (uint32_t a = 0; a < K; ++a)
        for (uint32_t b = 0; b < K; ++b) bd[P.trace_bonds_off + (s * K + a) * K + b] = bond(hist, K, P.hw, s, a, b);
  }
  static_cast<T*>(J.trace_obj)[g] = total;
  J.trace_id[g] = id;
}

// ACC (bit-mask path): kept configurations go to the warp's level accumulators while the list is
// unchanged; otherwise (and always with a shared-memory list) straight to the CTA table.
// ------------------------------------------------------------------------------ distinct configurations
// Exact key of the lane's configuration: per part, the rank of its species arrangement among all
// arrangements of the part's multiset (sites in order; arrangements that put a smaller species at the
// first differing site rank lower), combined over the parts in mixed radix. The host only enables
// keys when the product of the parts' arrangement counts is at most kDedupMaxSpace, so every
// intermediate M * c below stays under 2^48. The division M * c / n is exact: it is the number of
// arrangements of the remaining sites that start with species c's index.
static __device__ __noinline__ unsigned long long column_key(uint8_t* smem, const JobDesc& J, int t) {
  unsigned long long key = 0ull;
  for (uint32_t p = 0; p < J.n_parts; ++p) {
    const PartDesc& P = J.parts[p];
    const uint8_t* col = part_base(smem, P) + P.col_off + 4 * t;
    uint32_t c[kMaxSpecies];
    for (uint32_t k = 0; k < kMaxSpecies; ++k) c[k] = P.dd_counts[k];
    unsigned long long M = P.dd_space, r = 0ull;
    uint32_t n = P.n_sites;
    for (uint32_t x = 0; x < P.n_sites; ++x, --n) {
      const uint32_t sp = col[site_off(x)] >> 3;
      for (uint32_t k = 0; k < sp; ++k) r += M * c[k] / n;
      M = M * c[sp] / n;
      --c[sp];
    }
    key += r * P.dd_stride;
  }
  return key;
}

// Records (key, id, objective) in the job's distinct-configuration table: the first lane to bring a
// key claims a slot, and every lane with that key lowers the slot's id to the smallest. A key that
// finds no slot within kDedupProbes marks the record set incomplete (counters[kRecordsFull]).
static __device__ __noinline__ void dedup_insert(const JobDesc& J, unsigned long long key, unsigned long long id,
                                                 double objective) {
  unsigned long long h = mix64(key) & J.dedup_mask;
  for (int probe = 0; probe < kDedupProbes; ++probe, h = (h + 1) & J.dedup_mask) {
    DedupSlot& slot = J.dedup[h];
    const unsigned long long prev = atomicCAS(&slot.key, kDedupEmpty, key);
    if (prev == kDedupEmpty || prev == key) {
      atomicMin(&slot.id, id);
      slot.objective = objective;  // the same value from every lane with this key
      return;
    }
  }
  J.counters[kRecordsFull] = 1ull;
}

template <class T, bool ACC = false, class KeyF>
__device__ __forceinline__ void handle_candidates(const JobDesc& J, LevelSlot* ctab, WarpState& ws, bool pass, T total,
                                                  T thr_g, uint64_t id, int t, const KeyF& keyf) {
  const int lane = t & 31;
  unsigned m = __ballot_sync(0xffffffffu, pass);
  if (!m) return;
  const double v_mine = static_cast<double>(total);
  // Only values below the warp's (keep+1)-th entry that are not in its list yet change the list.
  bool fresh = pass && v_mine < ws.list_thr;
  int lo = 0;
  bool moved = false;
  const bool big = !ACC && ws.big != nullptr;  // warp-uniform; bit-mask jobs keep the register list (keep < 32)
  if (big) {
    if (__any_sync(0xffffffffu, fresh)) {
      const BigUpdate u = big_list_update(ws.big, ws.big_len, v_mine, fresh, J.keep, ws.list_thr);
      ws.list_thr = u.thr;
      moved = u.moved;
    }
  } else if (ACC || __any_sync(0xffffffffu, fresh)) {
    // Membership: the lower bound of each lane's value in the ascending list (one entry per lane),
    // found by a five-step shuffle search; then one insertion per distinct new value, lane order.
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const double e = __shfl_sync(0xffffffffu, ws.list, lo + step - 1);
      if (e < v_mine) lo += step;
    }
    const double at = __shfl_sync(0xffffffffu, ws.list, lo);  // every lane takes part in the shuffle
    fresh = fresh && at != v_mine;
    unsigned fm = __ballot_sync(0xffffffffu, fresh);
    moved = fm != 0;
    if (ACC && moved) warp_acc_flush(ws, ctab, J);  // list positions are about to move
    while (fm) {
      const double v = __shfl_sync(0xffffffffu, v_mine, __ffs(fm) - 1);
      fm &= ~__ballot_sync(0xffffffffu, v_mine == v);  // lanes with the same value: one insertion
      if (v < ws.list_thr) {
        const int pos = __popc(__ballot_sync(0xffffffffu, ws.list < v));
        const double up = __shfl_up_sync(0xffffffffu, ws.list, 1);
        if (lane == pos)
          ws.list = v;
        else if (lane > pos)
          ws.list = up;
        ws.list_thr = __shfl_sync(0xffffffffu, ws.list, J.keep);
      }
    }
  }
  if (lane == 0 && moved) {  // the bounds only change with the list
    const unsigned long long ot = ord_bits(ws.list_thr);
    if (ot < ws.published_thr) {
      atomicMin(&J.counters[kThreshold], ot);
      ws.published_thr = ot;
    }
    const unsigned long long ob = ord_bits(big ? ws.big[0] : ws.list);
    if (ob < ws.published_best) {
      atomicMin(&J.counters[kBest], ob);
      ws.published_best = ob;
    }
  }
  // The refreshed warp bound still dominates the final (keep+1)-th best, so it may filter.
  const double bound = fmin(ws.list_thr, static_cast<double>(thr_g));
  const bool keep_it = pass && v_mine <= bound;
  const unsigned km = __ballot_sync(0xffffffffu, keep_it);
  if (!km) return;
  if (ACC && !big && !moved) {
    // no insertion this step: a kept value (<= the (keep+1)-th entry) is in the list at lo
    if (keep_it) {
      const unsigned long long h = mix64(id);
      uint32_t* acc = warp_acc();
      atomicAdd(&acc[lo], 1u);
      atomicAdd(&acc[32 + lo], static_cast<unsigned>(h));
      atomicAdd(&acc[64 + lo], static_cast<unsigned>(h >> 32));
    }
  } else {
    // objective levels: one shared-memory update per distinct value per warp. The reductions run
    // with the full warp mask, one distinct value per round (a reduction whose mask differs between
    // the threads executing it is not allowed).
    const unsigned long long mykey = ord_bits(v_mine);
    const unsigned long long h = mix64(id);
    unsigned pending = km;
    while (pending) {
      const int leader = __ffs(pending) - 1;
      const unsigned long long key = __shfl_sync(0xffffffffu, mykey, leader);
      const bool in = keep_it && mykey == key;
      const unsigned gm = __ballot_sync(0xffffffffu, in);
      const unsigned sa = __reduce_add_sync(0xffffffffu, in ? static_cast<unsigned>(h) : 0u);
      const unsigned sb = __reduce_add_sync(0xffffffffu, in ? static_cast<unsigned>(h >> 32) : 0u);
      if (lane == leader) cta_level_add(ctab, J, key, __popc(gm), sa, sb);
      pending &= ~gm;
    }
  }
  if (J.dedup) {  // a deduplicating re-run: each distinct configuration once, with its smallest id
    if (keep_it) dedup_insert(J, keyf(), id, v_mine);
    return;
  }
  // Once the record buffer is full, appends stop (the level table stays exact) and the contended
  // candidate counter is left alone.
  unsigned long long base = 0;
  if (lane == 0) {
    if (ws.records_full ||
        *reinterpret_cast<volatile unsigned long long*>(&J.counters[kRecordsFull]) != 0ull) {
      ws.records_full = true;  // no more loads of the flag from this warp
      base = ~0ull;
    } else {
      base = atomicAdd(&J.counters[kCandidates], static_cast<unsigned long long>(__popc(km)));
      if (base + __popc(km) > J.capacity) {
        J.counters[kRecordsFull] = 1ull;
        ws.records_full = true;
      }
    }
  }
  base = __shfl_sync(0xffffffffu, base, 0);
  if (keep_it && base != ~0ull) {
    const uint64_t idx = base + __popc(km & ((1u << lane) - 1u));
    if (idx < J.capacity) reinterpret_cast<Cand*>(J.records)[idx] = Cand{v_mine, id};
  }
}

template <class T> __device__ __forceinline__ T load_threshold(const JobDesc& J) {
  const unsigned long long u = *reinterpret_cast<volatile unsigned long long*>(&J.counters[kThreshold]);
  return static_cast<T>(from_ord(u));
}

// ------------------------------------------------------------------------------ one tile
template <class T, int KW, bool SYS>
__device__ __forceinline__ void run_tile(const JobDesc& J, uint8_t* smem, LevelSlot* ctab, const Tile& tile,
                                      WarpState& ws) {
  using F = FP<T>;
  const int t = threadIdx.x;
  const uint64_t base = tile.count / kBlock, rem = tile.count % kBlock;
  const uint64_t my_count = base + (static_cast<uint64_t>(t) < rem ? 1 : 0);
  const uint64_t my_off = static_cast<uint64_t>(t) * base + min(static_cast<uint64_t>(t), rem);
  const uint64_t max_count = base + (rem ? 1 : 0);
  constexpr bool systematic = SYS;  // J.mode == 1
  // random mode: configuration id is the shuffle (shuffle_part) of the staged initial arrangement with
  // the words seeded by (seed, id) (shuffle_words); it depends on nothing but (seed, id), so any split
  // of the job into tiles, launches or devices evaluates the same configurations
  const uint32_t k0 = static_cast<uint32_t>(J.seed), k1 = static_cast<uint32_t>(J.seed >> 32);

  for (uint32_t p = 0; p < J.n_parts; ++p) init_column(smem, J.parts[p], t);
  uint32_t wlo = 0, wn = 0;
  if (systematic) {
    const PartDesc& P = J.parts[0];
    const uint32_t* win = reinterpret_cast<const uint32_t*>(part_base(smem, P) + P.win_off);
    wlo = win[0];
    wn = win[1] - win[0];
    if (my_count > 0)
      unrank_window(part_base(smem, P) + P.col_off + 4 * t, P, wlo, wn, tile.start + my_off, J.total);
  }
  T thr_g = load_threshold<T>(J);
  for (uint64_t it = 0; it < max_count; ++it) {
    const bool active = it < my_count;
    T total = T(0);
    if (active) {
      for (uint32_t p = 0; p < J.n_parts; ++p) {
        const PartDesc& P = J.parts[p];
        if (!systematic) {
          if (it > 0) init_column(smem, P, t);
          shuffle_part(smem, P, t, 0u, tile.start + my_off + it, p, k0, k1);
        }
        count_part<KW>(smem, J.blob, P, t);
        const T o = objective_part<T>(smem, P, t);
        total = p == 0 ? o : F::add(total, o);
      }
    }
    thr_g = load_threshold<T>(J);  // one L2 load per configuration: small next to its pair loop
    const double bound = fmin(ws.list_thr, static_cast<double>(thr_g));
    const bool pass = active && static_cast<double>(total) <= bound;
    const uint64_t id = tile.start + my_off + it;
    handle_candidates<T>(J, ctab, ws, pass, total, thr_g, id, t, [&] { return column_key(smem, J, t); });
    if (J.trace && active) write_trace<T>(J, smem, id - J.trace_base, total, id, t);
    if (systematic && active && it + 1 < my_count)
      next_permutation(part_base(smem, J.parts[0]) + J.parts[0].col_off + 4 * t, wlo, wn);
  }
}

// ------------------------------------------------------------------------------ binary fast path
// A configuration of a binary (K == 2) structure with N <= 64 sites is one word v: site x holds
// species 1 when bit N-1-x is set. The first site of a window is its most significant bit, so the
// lexicographic order of core/permutation.h:80-102 is the integer order and next_permutation is the
// next larger word with the same popcount (Gosper's hack). With NB_s[i] the mask of the sites j > i
// in shell s and b_i the species of site i,
//   D = sum_i popc(NB_s[i] & v)      = n(s,1,1) + n(s,0,1)
//   A = sum_i b_i popc(NB_s[i] & v)  = n(s,1,1)
//   E = sum_i b_i popc(NB_s[i])      = n(s,1,1) + n(s,1,0)
// and n(s,0,0) = P_s minus the rest: the ordered counts of optimization.h:74-77, exactly. The
// draws (Fisher-Yates swaps, or Floyd's sampling on a two-species window) and the visiting order are
// the general path's, so both evaluate the same configurations for a job.
template <int W> struct Word;
template <> struct Word<1> {
  using type = uint32_t;
  static __device__ __forceinline__ uint32_t pc(type v, uint32_t lo, uint32_t) { return __popc(v & lo); }
  // trailing zeros of v != 0 as one popcount (a find-first-set is a bit reverse plus a leading-zero count)
  static __device__ __forceinline__ int ctz(type v) { return __popc(~v & (v - 1)); }
};
template <> struct Word<2> {
  using type = unsigned long long;
  static __device__ __forceinline__ uint32_t pc(type v, uint32_t lo, uint32_t hi) {
    return __popc(static_cast<uint32_t>(v) & lo) + __popc(static_cast<uint32_t>(v >> 32) & hi);
  }
  static __device__ __forceinline__ int ctz(type v) { return __popcll(~v & (v - 1)); }  // v != 0
};

template <class V> __device__ __forceinline__ V low_mask(uint32_t n) {
  return n >= sizeof(V) * 8 ? ~V(0) : ((V(1) << n) - V(1));
}

// Ordered bond counts of shell s for word v.
template <class V, int W>
__device__ __forceinline__ void k2_counts(const uint4* ent, uint32_t e0, uint32_t e1, uint32_t ps, V v,
                                          uint32_t& n00, uint32_t& n01, uint32_t& n10, uint32_t& n11) {
  uint32_t A = 0, D = 0, E = 0;
  for (uint32_t e = e0; e < e1; ++e) {
    const uint4 q = ent[e];
    const uint32_t c = Word<W>::pc(v, q.x, q.y);
    const uint32_t b = static_cast<uint32_t>(v >> q.z) & 1u;
    D += c;
    A += b * c;
    E += b * q.w;
  }
  n11 = A;
  n01 = D - A;
  n10 = E - A;
  n00 = ps - n11 - n01 - n10;
}

// popc(NB_s[site of bit bp] & u) from the bit-position table (u32 entries for N <= 32: the lanes'
// different positions fall in different banks; uint2 entries otherwise).
template <class V, int W>
__device__ __forceinline__ uint32_t k2_nbp_count(const uint8_t* tab, int s, int bp, V u) {
  if (W == 1) {
    const uint32_t m = reinterpret_cast<const uint32_t*>(tab)[s * 32 + bp];
    return __popc(static_cast<uint32_t>(u) & m);
  } else {
    const uint2 m = reinterpret_cast<const uint2*>(tab)[s * 64 + bp];
    return Word<W>::pc(u, m.x, m.y);
  }
}

// Pairs inside the minority species (the nb set bits x of vv), shell by shell, for NS shells. Every
// configuration of a job has the same nb, so the loop is counted and unrolled: the scheduler sees
// several bits' loads and popcounts at once.
template <class V, int W, int NS>
__device__ __forceinline__ void k2_minority_pairs(const uint8_t* nbp, V vv, V x, uint32_t* a, int nb) {
#pragma unroll 4
  for (int k = 0; k < nb; ++k) {  // the loop-carried chain (x &= x - 1) stays off the popcount unit
    const int bp = Word<W>::ctz(x);
    x &= x - 1;
#pragma unroll
    for (int s = 0; s < NS; ++s) a[s] += k2_nbp_count<V, W>(nbp, s, bp, vv);
  }
}

// What the objective needs per shell: n11, n01 + n10 and n00. With deg_s(x) the number of shell-s
// pairs at site x, sum_x b_x deg_s(x) = 2 n11 + n01 + n10 (the degree classes, sites of equal degree
// as one mask, give it in one popcount per class but the largest, whose share follows from the fixed
// number of ones) and sum_x deg_s(x) = 2 P_s, so one count of the pairs inside the minority species
// fixes all three.

template <class T>
__device__ __forceinline__ T k2_term(T obj, uint32_t n, const T* f, const T* w, const T* tg, uint32_t d) {
  using F = FP<T>;
  const T sig = F::sub(T(1), F::mul(F::cvt(n), f[d]));
  T diff = F::sub(sig, tg[d]);
  diff = diff > T(0) ? diff : -diff;
  return F::add(obj, F::mul(w[d], diff));
}

// Writes the lane's species codes and bond histogram like the general path keeps them, so that the
// general record and trace writers can be used.
template <class V, int W>
__device__ __forceinline__ void k2_materialize(uint8_t* smem, const PartDesc& P, int t, V v) {
  uint8_t* part = part_base(smem, P);
  uint8_t* col = part + P.col_off + 4 * t;
  uint32_t* hist = reinterpret_cast<uint32_t*>(part + P.hist_off) + t;
  const uint32_t N = P.n_sites;
  for (uint32_t x = 0; x < N; ++x) col[site_off(x)] = static_cast<uint8_t>((static_cast<uint32_t>(v >> (N - 1 - x)) & 1u) << 3);
  const uint4* ent = reinterpret_cast<const uint4*>(part + P.k2_off);
  const uint32_t* sh = reinterpret_cast<const uint32_t*>(part + P.k2_shell_off);
  uint32_t e0 = 0;
  for (uint32_t s = 0; s < P.n_shells; ++s) {
    uint32_t n00, n01, n10, n11;
    k2_counts<V, W>(ent, e0, sh[8 * s + 1], sh[8 * s], v, n00, n01, n10, n11);
    e0 = sh[8 * s + 1];
    hist[(s * 2 + 0) * kBlock] = n00 | (n01 << 16);
    hist[(s * 2 + 1) * kBlock] = n10 | (n11 << 16);
  }
}

template <class T, int W, bool SYS>
__device__ __forceinline__ void run_tile_k2(const JobDesc& J, uint8_t* smem, LevelSlot* ctab, const Tile& tile,
                                         WarpState& ws) {
  using V = typename Word<W>::type;
  const int t = threadIdx.x;
  const PartDesc& P = J.parts[0];
  const uint64_t base = tile.count / kBlock, rem = tile.count % kBlock;
  const uint64_t my_count = base + (static_cast<uint64_t>(t) < rem ? 1 : 0);
  const uint64_t my_off = static_cast<uint64_t>(t) * base + min(static_cast<uint64_t>(t), rem);
  const uint64_t max_count = base + (rem ? 1 : 0);
  constexpr bool systematic = SYS;  // J.mode == 1
  const uint32_t k0 = static_cast<uint32_t>(J.seed), k1 = static_cast<uint32_t>(J.seed >> 32);
  const uint8_t* part = part_base(smem, P);
  const uint32_t N = P.n_sites, S = P.n_shells;
  const uint4* ent = reinterpret_cast<const uint4*>(part + P.k2_off);
  const uint32_t* sh = reinterpret_cast<const uint32_t*>(part + P.k2_shell_off);
  const T* f = reinterpret_cast<const T*>(part + P.cube_off);
  const T* w = f + 4 * S;
  const T* tg = w + 4 * S;
  const uint32_t* win = reinterpret_cast<const uint32_t*>(part + P.win_off);
  V v0 = 0;  // the staged initial arrangement (random jobs: the other species on each Floyd window)
  for (uint32_t x = 0; x < N; ++x)
    if (part[P.species_off + x]) v0 |= V(1) << (N - 1 - x);
  // minority sites: the same number in every configuration (shuffles keep the composition; the staged
  // arrangement of a random job holds only the other species on its Floyd windows)
  const int nb = static_cast<int>(P.k2_zeros ? N - P.ones : P.ones);
  V v = v0;
  uint32_t wn = 0, wshift = 0;
  V wmask = 0;
  if (systematic) {
    wn = win[1] - win[0];
    wshift = N - win[1];
    wmask = low_mask<V>(wn) << wshift;
    if (my_count > 0) {
      // core/permutation.h:52-78 for two species: the arrangements of the remaining m positions that
      // start with species 0 number total*h0/m = C(m-1, h1), read from the job's binomial table.
      const unsigned long long* binom = reinterpret_cast<const unsigned long long*>(J.blob + P.k2_binom_off);
      const uint32_t cols = P.unrank_hist[1] + 1;
      uint64_t rank = tile.start + my_off;
      uint32_t h1 = P.unrank_hist[1];
      V word = 0;
      for (uint32_t k = 0; k < wn; ++k) {
        const uint32_t m = wn - k;
        const uint64_t s0 = h1 <= m - 1 ? __ldg(&binom[(m - 1) * cols + h1]) : 0ull;
        if (rank > s0) {
          rank -= s0;
          --h1;
          word |= V(1) << (wn - 1 - k);
        }
      }
      v = (v & ~wmask) | (word << wshift);
    }
  }
  T thr_g = load_threshold<T>(J);
  for (uint64_t it = 0; it < max_count; ++it) {
    const bool active = it < my_count;
    T total = T(0);
    if (active) {
      if (!systematic) {  // core/shuffle.h:39-50 on bits, the same words as the general path
        const uint64_t cid = tile.start + my_off + it;
        xoshiro128ss words =
            shuffle_words(0u, static_cast<uint32_t>(cid), static_cast<uint32_t>(cid >> 32) << 8, k0, k1);
        v = v0;
        for (uint32_t wi = 0; wi < P.n_windows; ++wi) {
          const uint32_t lo = win[2 * wi], n = win[2 * wi + 1] - lo, fw = win[2 * P.n_windows + wi];
          const uint32_t top = N - 1 - lo;  // bit of the window's first site
          if (fw) {  // floyd_window on bits: the window holds the other species, flip the drawn sites
            const V rare = (fw >> 16) & 0xffu ? V(1) : V(0);
            for (uint32_t j = n - (fw & 0xffffu); j < n; ++j) {
              const uint32_t bt = top - __umulhi(words.next(), j + 1);
              v ^= V(1) << (((v >> bt) & V(1)) == rare ? top - j : bt);
            }
          } else {
            for (uint32_t i = n; i > 1; --i) {
              const uint32_t pp = __umulhi(words.next(), i);
              const uint32_t ba = top - (i - 1), bb = top - pp;
              const V dlt = ((v >> ba) ^ (v >> bb)) & V(1);
              v ^= (dlt << ba) | (dlt << bb);
            }
          }
        }
      }
      // pairs within the minority species, for up to kK2MaxShells shells in one pass over its set
      // bits (every lane has the same number of them: no divergence)
      const V vv = P.k2_zeros ? ~v : v;
      V x = vv & low_mask<V>(N);
      uint32_t a[kK2MaxShells] = {};
      const uint8_t* nbp = part + P.k2_nbp_off;
      switch (S) {  // one copy of the loop per shell count: no predicated work for absent shells
        case 1: k2_minority_pairs<V, W, 1>(nbp, vv, x, a, nb); break;
        case 2: k2_minority_pairs<V, W, 2>(nbp, vv, x, a, nb); break;
        case 3: k2_minority_pairs<V, W, 3>(nbp, vv, x, a, nb); break;
        default: k2_minority_pairs<V, W, 4>(nbp, vv, x, a, nb); break;
      }
#pragma unroll
      for (int s = 0; s < kK2MaxShells; ++s) {
        if (s >= static_cast<int>(S)) break;
        uint32_t DE = sh[8 * s + 4];  // sum over the ones of their shell-s degree: 2 n11 + n01 + n10
        for (uint32_t e = sh[8 * s + 2]; e < sh[8 * s + 3]; ++e) {
          const uint4 q = ent[e];
          DE += q.z * Word<W>::pc(v, q.x, q.y);
        }
        const uint32_t ps = sh[8 * s];
        uint32_t n00, nx, n11;
        if (P.k2_zeros) {
          n00 = a[s];
          nx = (2u * ps - DE) - 2u * n00;
          n11 = ps - n00 - nx;
        } else {
          n11 = a[s];
          nx = DE - 2u * n11;
          n00 = ps - n11 - nx;
        }
        total = k2_term<T>(total, n00, f, w, tg, s * 4 + 0);
        total = k2_term<T>(total, nx, f, w, tg, s * 4 + 1);
        total = k2_term<T>(total, n11, f, w, tg, s * 4 + 3);
      }
    }
    if ((it & 15) == 0) thr_g = load_threshold<T>(J);
    const double bound = fmin(ws.list_thr, static_cast<double>(thr_g));
    const bool pass = active && static_cast<double>(total) <= bound;
    const uint64_t id = tile.start + my_off + it;
    handle_candidates<T, true>(J, ctab, ws, pass, total, thr_g, id, t,
                               [&] { return static_cast<unsigned long long>(v); });
    if (J.trace && active) {
      k2_materialize<V, W>(smem, P, t, v);
      write_trace<T>(J, smem, id - J.trace_base, total, id, t);
    }
    if (systematic && active && it + 1 < my_count) {  // Gosper's hack inside the window
      const V x = (v & wmask) >> wshift;
      const V tt = x | (x - 1);
      const V nx = (tt + 1) | (((~tt & (tt + 1)) - 1) >> (Word<W>::ctz(x) + 1));
      v = (v & ~wmask) | ((nx << wshift) & wmask);
    }
  }
  warp_acc_flush(ws, ctab, J);  // the CTA table is complete for this tile
}

// ------------------------------------------------------------------------------ lattice path
// A supercell of A x B x C copies of a unit cell with m sites: site (beta, c) is unit-cell site beta
// in cell c = x + A*(y + B*z). Translating every site by one cell vector maps the pair list onto
// itself (distances and shells depend only on the difference vector), so the pairs of one shell fall
// into classes {(beta, c), (beta2, c + d)} over all cells c. With X[beta][a] the set of cells whose
// site beta holds species a (W 64-bit words: up to 64 or 128 cells), the pairs of one class with
// species {a, b} number
//   popc(X[beta][a] & Y[b]) + popc(X[beta][b] & Y[a]),  Y[b] = X[beta2][b] translated by -d,
// (one popcount of the OR: the two sets are disjoint), and a class that is its own reverse
// (beta == beta2, 2d = 0) counts each pair twice. Counting only the species a, b < K-1 and closing with
// the degree identity sum_b (1 + [a == b]) U(a, b) = sum_{sites i of species a} deg_s(i) gives the
// unordered counts U(a, b) = bonds(s,a,b) + bonds(s,b,a) (a != b) and U(a, a) = bonds(s,a,a) that
// core/optimization.h:79-103 reads, exactly. A class costs one AND (+ OR) and one popcount per
// species pair and word instead of one gather per pair of sites.

// W-word cell sets; shifts by 0 < k < 64 W (a warp-uniform amount: one translation for all lanes).
template <int W> struct LatBits {
  unsigned long long w[W];
};

template <int W> __device__ __forceinline__ LatBits<W> lat_shl(const LatBits<W>& v, uint32_t k) {
  LatBits<W> r;
  if constexpr (W == 1) {
    r.w[0] = v.w[0] << k;
  } else {
    if (k >= 64) {
      r.w[1] = v.w[0] << (k - 64);
      r.w[0] = 0ull;
    } else {
      r.w[1] = (v.w[1] << k) | (v.w[0] >> (64 - k));
      r.w[0] = v.w[0] << k;
    }
  }
  return r;
}

template <int W> __device__ __forceinline__ LatBits<W> lat_shr(const LatBits<W>& v, uint32_t k) {
  LatBits<W> r;
  if constexpr (W == 1) {
    r.w[0] = v.w[0] >> k;
  } else {
    if (k >= 64) {
      r.w[0] = v.w[1] >> (k - 64);
      r.w[1] = 0ull;
    } else {
      r.w[0] = (v.w[0] >> k) | (v.w[1] << (64 - k));
      r.w[1] = v.w[1] >> k;
    }
  }
  return r;
}

// Translation of a cell set by (tx, ty, tz): rotations inside rows of A bits, blocks of A*B bits and
// the whole grid of A*B*C bits; a zero shift skips its stage. mxh, myh mark the cells whose source does
// not wrap (taken from the left shift); the others take the right shift. Outside the grid a set has
// no bits and the right shifts bring in none (their sources lie past the grid), so one select per
// word, a single three-input logic op, blends the two shifts.
template <int W>
__device__ __forceinline__ LatBits<W> lat_translate(LatBits<W> v, const LatTrW<W>* t, const LatBits<W>& full) {
  if (t->sx) {
    const LatBits<W> h = lat_shl<W>(v, t->sx), l = lat_shr<W>(v, t->sxr);
#pragma unroll
    for (int k = 0; k < W; ++k) v.w[k] = (h.w[k] & t->mxh[k]) | (l.w[k] & ~t->mxh[k]);
  }
  if (t->sy) {
    const LatBits<W> h = lat_shl<W>(v, t->sy), l = lat_shr<W>(v, t->syr);
#pragma unroll
    for (int k = 0; k < W; ++k) v.w[k] = (h.w[k] & t->myh[k]) | (l.w[k] & ~t->myh[k]);
  }
  if (t->sz) {
    const LatBits<W> h = lat_shl<W>(v, t->sz), l = lat_shr<W>(v, t->szr);
#pragma unroll
    for (int k = 0; k < W; ++k) v.w[k] = (h.w[k] | l.w[k]) & full.w[k];
  }
  return v;
}

template <int W> __device__ __forceinline__ LatBits<W> lat_full(const PartDesc& P) {
  LatBits<W> f;
  f.w[0] = P.lat_full;
  if constexpr (W == 2) f.w[1] = P.lat_full_hi;
  return f;
}

// Plane (beta, a) of lane t: W words at [(beta * (K-1) + a) * W + k] * kBlock + t.
template <int W>
__device__ __forceinline__ LatBits<W> lat_load(const unsigned long long* X, uint32_t plane) {
  LatBits<W> v;
#pragma unroll
  for (int k = 0; k < W; ++k) v.w[k] = X[(plane * W + k) * kBlock];
  return v;
}

// The lane's one-hot planes X[beta][a] (a < K-1) from its species column: four sites per step, bit k
// of each site's species gathered into a nibble (binary planes), then one-hot by AND/NOT.
template <int KM, int W>
__device__ __forceinline__ void lat_planes(uint8_t* smem, const PartDesc& P, int t) {
  uint8_t* part = part_base(smem, P);
  const uint8_t* col = part + P.col_off + 4 * t;
  const uint4* so4 = reinterpret_cast<const uint4*>(part + P.lat_site_off);
  unsigned long long* X = reinterpret_cast<unsigned long long*>(part + P.lat_planes_off) + t;
  const uint32_t km1 = P.n_species - 1, chunks = P.lat_chunks;
  const LatBits<W> full = lat_full<W>(P);
  constexpr int NB = KM <= 2 ? 1 : (KM <= 4 ? 2 : 3);
  for (uint32_t beta = 0; beta < P.lat_basis; ++beta) {
    unsigned long long B[NB][W];
#pragma unroll
    for (int k = 0; k < NB; ++k)
#pragma unroll
      for (int w = 0; w < W; ++w) B[k][w] = 0ull;
    for (uint32_t q = 0; q < chunks; ++q) {
      const uint4 o = so4[beta * chunks + q];
      const uint32_t w4 = static_cast<uint32_t>(col[o.x]) | (static_cast<uint32_t>(col[o.y]) << 8) |
                          (static_cast<uint32_t>(col[o.z]) << 16) | (static_cast<uint32_t>(col[o.w]) << 24);
#pragma unroll
      for (int k = 0; k < NB; ++k) {  // species codes are 8 * species: bit k of the species is bit 3 + k
        const unsigned long long nib = ((((w4 >> (3 + k)) & 0x01010101u) * 0x00204081u) >> 21) & 0xfu;
        if constexpr (W == 1) {
          B[k][0] |= nib << (4 * q);
        } else {
          if (q < 16)
            B[k][0] |= nib << (4 * q);
          else
            B[k][1] |= nib << (4 * (q - 16));
        }
      }
    }
#pragma unroll
    for (int a = 0; a < KM - 1; ++a) {
      if (a >= static_cast<int>(km1)) break;
#pragma unroll
      for (int w = 0; w < W; ++w) {
        unsigned long long x = full.w[w];
#pragma unroll
        for (int k = 0; k < NB; ++k) x &= ((a >> k) & 1) ? B[k][w] : ~B[k][w];
        X[((beta * km1 + a) * W + w) * kBlock] = x;
      }
    }
  }
}

template <int NA> __host__ __device__ constexpr int lat_idx(int a, int b) { return a * NA - a * (a - 1) / 2 + (b - a); }

template <int W> __device__ __forceinline__ uint32_t lat_popc(const LatBits<W>& v) {
  uint32_t c = 0;
#pragma unroll
  for (int k = 0; k < W; ++k) c += __popcll(v.w[k]);
  return c;
}

// Objective of one part (core/optimization.h:79-103, terms in the reference's order) from the lane's
// planes.
template <int KM, class T, int W>
__device__ __forceinline__ T lat_objective(uint8_t* smem, const PartDesc& P, int t) {
  using F = FP<T>;
  constexpr int NA = KM - 1;  // species with planes, at most
  constexpr int NT = NA * (NA + 1) / 2;
  const uint8_t* part = part_base(smem, P);
  const unsigned long long* X = reinterpret_cast<const unsigned long long*>(part + P.lat_planes_off) + t;
  const uint32_t* ent = reinterpret_cast<const uint32_t*>(part + P.lat_ent_off);
  const uint4* shl = reinterpret_cast<const uint4*>(part + P.lat_shell_off);
  const LatTrW<W>* trs = reinterpret_cast<const LatTrW<W>*>(part + P.lat_tr_off);
  const uint32_t* deg = reinterpret_cast<const uint32_t*>(part + P.lat_deg_off);
  const uint32_t K = P.n_species, km1 = K - 1, S = P.n_shells, m = P.lat_basis;
  const LatBits<W> full = lat_full<W>(P);
  const uint32_t skk = S * K * K;
  const T* f = reinterpret_cast<const T*>(part + P.cube_off);
  const T* w = f + skk;
  const T* tg = w + skk;
  T obj = T(0);
  for (uint32_t s = 0; s < S; ++s) {
    uint32_t acc[NT];
#pragma unroll
    for (int k = 0; k < NT; ++k) acc[k] = 0u;
    const uint4 sh = shl[s];
    uint32_t key = ~0u, cur = ~0u;
    LatBits<W> Y[NA], Xa[NA];
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int k = 0; k < W; ++k) Y[a].w[k] = Xa[a].w[k] = 0ull;
    for (uint32_t e = sh.x; e < sh.z; ++e) {
      if (e == sh.y) {  // self-reverse classes count every pair twice: double what came before
#pragma unroll
        for (int k = 0; k < NT; ++k) acc[k] <<= 1;
      }
      const uint32_t en = ent[e];
      if ((en >> 4) != key) {  // (beta2, translation) changed: translate beta2's planes
        key = en >> 4;
        const uint32_t b2 = key & 0xfu;
        const LatTrW<W>* tr = trs + (key >> 4);
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          if (a >= static_cast<int>(km1)) break;
          Y[a] = lat_translate<W>(lat_load<W>(X, b2 * km1 + a), tr, full);
        }
      }
      if ((en & 0xfu) != cur) {
        cur = en & 0xfu;
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          if (a >= static_cast<int>(km1)) break;
          Xa[a] = lat_load<W>(X, cur * km1 + a);
        }
      }
#pragma unroll
      for (int a = 0; a < NA; ++a) {
#pragma unroll
        for (int b = a; b < NA; ++b) {
          if (b >= static_cast<int>(km1)) break;
          uint32_t c = 0;
#pragma unroll
          for (int k = 0; k < W; ++k)
            c += a == b ? __popcll(Xa[a].w[k] & Y[a].w[k])
                        : __popcll((Xa[a].w[k] & Y[b].w[k]) | (Xa[b].w[k] & Y[a].w[k]));
          acc[lat_idx<NA>(a, b)] += c;
        }
      }
    }
    if (sh.y < sh.z) {
#pragma unroll
      for (int k = 0; k < NT; ++k) acc[k] >>= 1;
    }
    // pairs with the last species: H_a - 2 U(a, a) - sum_{b != a} U(a, b), H_a the shell-s degree sum
    // of the sites of species a; U(K-1, K-1) from the shell's pair count
    uint32_t ue[NA];
    uint32_t rest = sh.w;
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      ue[a] = 0u;
      if (a >= static_cast<int>(km1)) break;
      uint32_t h = 0u;
      for (uint32_t beta = 0; beta < m; ++beta) h += deg[s * m + beta] * lat_popc<W>(lat_load<W>(X, beta * km1 + a));
      uint32_t u = h - 2u * acc[lat_idx<NA>(a, a)];
#pragma unroll
      for (int b = 0; b < NA; ++b) {
        if (b >= static_cast<int>(km1)) break;
        if (b != a) u -= acc[b < a ? lat_idx<NA>(b, a) : lat_idx<NA>(a, b)];
      }
      ue[a] = u;
      rest -= u;
#pragma unroll
      for (int b = a; b < NA; ++b) {
        if (b >= static_cast<int>(km1)) break;
        rest -= acc[lat_idx<NA>(a, b)];
      }
    }
    const uint32_t uee = rest;
#pragma unroll
    for (int xi = 0; xi < KM; ++xi) {
      if (xi >= static_cast<int>(K)) break;
      const int xc = xi < NA ? xi : 0;
      const uint32_t d = (s * K + xi) * K + xi;
      const uint32_t nd = static_cast<uint32_t>(xi) == km1 ? uee : (xi < NA ? acc[lat_idx<NA>(xc, xc)] : 0u);
      const T sig = F::sub(T(1), F::mul(F::cvt(nd), f[d]));
      T diff = F::sub(sig, tg[d]);
      diff = diff > T(0) ? diff : -diff;
      obj = F::add(obj, F::mul(w[d], diff));
#pragma unroll
      for (int eta = xi + 1; eta < KM; ++eta) {
        if (eta >= static_cast<int>(K)) break;
        const int ec = eta < NA ? eta : 0;
        const uint32_t u = (s * K + xi) * K + eta;
        const uint32_t nb = static_cast<uint32_t>(eta) == km1 ? (xi < NA ? ue[xc] : 0u)
                                                              : (eta < NA ? acc[lat_idx<NA>(xc, ec)] : 0u);
        const T sg = F::sub(T(1), F::mul(F::cvt(nb), f[u]));
        T df = F::sub(sg, tg[u]);
        df = df > T(0) ? df : -df;
        obj = F::add(obj, F::mul(w[u], df));
      }
    }
  }
  return obj;
}

// One variant per unrolled species count up to the kernel's KMAX (a kernel holds only the variants
// it may meet, so that its register budget is that of its largest variant).
template <class T, int KMAX, int W>
__device__ __forceinline__ T lat_part(uint8_t* smem, const PartDesc& P, int t) {
  if (P.lat_km == 2) {
    lat_planes<2, W>(smem, P, t);
    return lat_objective<2, T, W>(smem, P, t);
  }
  if constexpr (KMAX >= 3) {
    if (P.lat_km == 3) {
      lat_planes<3, W>(smem, P, t);
      return lat_objective<3, T, W>(smem, P, t);
    }
  }
  if constexpr (KMAX >= 4) {
    if (P.lat_km == 4) {
      lat_planes<4, W>(smem, P, t);
      return lat_objective<4, T, W>(smem, P, t);
    }
  }
  if constexpr (KMAX >= 5) {
    if (P.lat_km == 5) {
      lat_planes<5, W>(smem, P, t);
      return lat_objective<5, T, W>(smem, P, t);
    }
  }
  if constexpr (KMAX >= 8) {
    lat_planes<8, W>(smem, P, t);
    return lat_objective<8, T, W>(smem, P, t);
  }
  return T(0);  // not reached: the host launches a job only in a kernel with KMAX >= its lat_kmax
}

// The general tile loop with lattice counting. In trace mode the pair-stream count runs as well: its
// ordered bonds go to the trace, and an objective that differs from the lattice path's is counted in
// counters[kMismatch] (the host reports it as an error).
template <class T, bool SYS, int KMAX, int W>
__device__ __forceinline__ void run_tile_lat(const JobDesc& J, uint8_t* smem, LevelSlot* ctab, const Tile& tile,
                                             WarpState& ws) {
  using F = FP<T>;
  const int t = threadIdx.x;
  const uint64_t base = tile.count / kBlock, rem = tile.count % kBlock;
  const uint64_t my_count = base + (static_cast<uint64_t>(t) < rem ? 1 : 0);
  const uint64_t my_off = static_cast<uint64_t>(t) * base + min(static_cast<uint64_t>(t), rem);
  const uint64_t max_count = base + (rem ? 1 : 0);
  const uint32_t k0 = static_cast<uint32_t>(J.seed), k1 = static_cast<uint32_t>(J.seed >> 32);
  for (uint32_t p = 0; p < J.n_parts; ++p) init_column(smem, J.parts[p], t);
  uint32_t wlo = 0, wn = 0;
  if (SYS) {
    const PartDesc& P = J.parts[0];
    const uint32_t* win = reinterpret_cast<const uint32_t*>(part_base(smem, P) + P.win_off);
    wlo = win[0];
    wn = win[1] - win[0];
    if (my_count > 0)
      unrank_window(part_base(smem, P) + P.col_off + 4 * t, P, wlo, wn, tile.start + my_off, J.total);
  }
  T thr_g = load_threshold<T>(J);
  for (uint64_t it = 0; it < max_count; ++it) {
    const bool active = it < my_count;
    T total = T(0);
    if (active) {
      for (uint32_t p = 0; p < J.n_parts; ++p) {
        const PartDesc& P = J.parts[p];
        if (!SYS) {
          if (it > 0) init_column(smem, P, t);
          shuffle_part(smem, P, t, 0u, tile.start + my_off + it, p, k0, k1);
        }
        const T o = lat_part<T, KMAX, W>(smem, P, t);
        if (J.trace) {
          if (J.kw == 1)
            count_part<1>(smem, J.blob, P, t);
          else
            count_part<2>(smem, J.blob, P, t);
          const T g = objective_part<T>(smem, P, t);
          if (!(g == o)) atomicAdd(&J.counters[kMismatch], 1ull);
        }
        total = p == 0 ? o : F::add(total, o);
      }
    }
    thr_g = load_threshold<T>(J);
    const double bound = fmin(ws.list_thr, static_cast<double>(thr_g));
    const bool pass = active && static_cast<double>(total) <= bound;
    const uint64_t id = tile.start + my_off + it;
    handle_candidates<T>(J, ctab, ws, pass, total, thr_g, id, t, [&] { return column_key(smem, J, t); });
    if (J.trace && active) write_trace<T>(J, smem, id - J.trace_base, total, id, t);
    if (SYS && active && it + 1 < my_count)
      next_permutation(part_base(smem, J.parts[0]) + J.parts[0].col_off + 4 * t, wlo, wn);
  }
}

// ------------------------------------------------------------------------------ persistent kernel
constexpr unsigned long long kNoTile = ~0ull;

// Live mode: claim the next published ring entry, waiting (bounded) for the host to publish more.
__device__ __forceinline__ uint32_t sm_id() {
  uint32_t id;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(id));
  return id;
}

// Live mode: may this CTA work on its SM for its ring?
__device__ __forceinline__ bool owns_sm(const QueueCtl* q, uint32_t smid) {
  if (q->n_owner == 0) return true;
  return smid < q->n_owner && q->owner[smid] == q->ring;
}

__device__ __forceinline__ unsigned long long claim_live(QueueCtl* q, const volatile int32_t* cancel, uint32_t smid) {
  uint32_t idle = 0;
  for (;;) {
    if (!owns_sm(q, smid)) return kNoTile;  // the SM went to another ring
    // a pending yield unit ends this CTA (each loop round takes one unit or sees another CTA take it)
    uint32_t y = *reinterpret_cast<volatile unsigned int*>(&q->yield);
    while (y != 0) {
      const uint32_t o = atomicCAS(&q->yield, y, y - 1);
      if (o == y) return kNoTile;
      y = o;
    }
    const unsigned long long tl = *reinterpret_cast<volatile unsigned long long*>(&q->tail);
    const unsigned long long hd = *reinterpret_cast<volatile unsigned long long*>(&q->head);
    if (hd < tl) {
      if (atomicCAS(&q->head, hd, hd + 1) == hd) {
        __threadfence();  // the tile and its job's descriptor were written before tail was raised
        return hd;
      }
      continue;  // another CTA took tile hd
    }
    if ((cancel && *cancel) || ++idle > q->idle_limit) return kNoTile;
    __nanosleep(2000);
  }
}

// One instantiation per (path, precision, row width, mode): random and systematic loops keep only
// their own state live.
template <bool SYS>
__device__ __forceinline__ void dispatch_mask(const JobDesc& sj, uint8_t* smem, LevelSlot* ctab, const Tile& tile,
                                              WarpState& ws) {
  if (sj.k2 == 1) {
    if (sj.prec == 1)
      run_tile_k2<double, 1, SYS>(sj, smem, ctab, tile, ws);
    else
      run_tile_k2<float, 1, SYS>(sj, smem, ctab, tile, ws);
  } else if (sj.k2 == 2) {
    if (sj.prec == 1)
      run_tile_k2<double, 2, SYS>(sj, smem, ctab, tile, ws);
    else
      run_tile_k2<float, 2, SYS>(sj, smem, ctab, tile, ws);
  }
}

// Reference-stream debug mode (random jobs, general path): each thread runs one of the reference's
// thread-pool blocks as a chain, like its single worker thread does (sqs.h:348-455 with one thread):
// the block starts from the packed arrangement (sqs.h:374) and the part's stream at the block's state;
// interact mode evaluates, then shuffles (sqs.h:397-403,439-440); split mode shuffles every part,
// then evaluates it (sqs.h:404-413). A tile is up to 128 consecutive blocks; configuration ids are
// the reference's iteration indices.
template <class T, int KW>
__device__ __forceinline__ void run_tile_chain(const JobDesc& J, uint8_t* smem, LevelSlot* ctab, const Tile& tile,
                                               WarpState& ws) {
  using F = FP<T>;
  const int t = threadIdx.x;
  const bool mine = static_cast<uint64_t>(t) < tile.count;
  const uint64_t b = tile.start + static_cast<uint64_t>(t);
  const uint64_t first = mine ? chain_block_start(J, b) : 0, last = mine ? chain_block_end(J, b) : 0;
  unsigned long long st[kMaxParts];
  for (uint32_t p = 0; p < J.n_parts; ++p) {
    init_column(smem, J.parts[p], t);
    st[p] = chain_state(J, J.parts[p], first);
  }
  T thr_g = load_threshold<T>(J);
  // every lane steps through the longest block (chain_block + 1): the candidate steps are warp-wide
  for (uint64_t j = 0; j <= J.chain_block; ++j) {
    const uint64_t id = first + j;
    const bool active = mine && id < last;
    T total = T(0);
    if (active) {
      for (uint32_t p = 0; p < J.n_parts; ++p) {
        const PartDesc& P = J.parts[p];
        if (J.chain_split) shuffle_part_rapid(smem, P, t, st[p]);
        count_part<KW>(smem, J.blob, P, t);
        const T o = objective_part<T>(smem, P, t);
        total = p == 0 ? o : F::add(total, o);
      }
    }
    if ((j & 15) == 0) thr_g = load_threshold<T>(J);
    const double bound = fmin(ws.list_thr, static_cast<double>(thr_g));
    const bool pass = active && static_cast<double>(total) <= bound;
    handle_candidates<T>(J, ctab, ws, pass, total, thr_g, id, t, [&] { return column_key(smem, J, t); });
    if (J.trace && active) write_trace<T>(J, smem, id - J.trace_base, total, id, t);
    if (active && !J.chain_split) shuffle_part_rapid(smem, J.parts[0], t, st[0]);
  }
}

template <bool SYS, int KMAX, int W>
__device__ __forceinline__ void dispatch_lattice(const JobDesc& sj, uint8_t* smem, LevelSlot* ctab, const Tile& tile,
                                                 WarpState& ws) {
  if (sj.prec == 1)
    run_tile_lat<double, SYS, KMAX, W>(sj, smem, ctab, tile, ws);
  else
    run_tile_lat<float, SYS, KMAX, W>(sj, smem, ctab, tile, ws);
}

template <bool SYS>
__device__ __forceinline__ void dispatch_general(const JobDesc& sj, uint8_t* smem, LevelSlot* ctab, const Tile& tile,
                                                 WarpState& ws) {
  if (!SYS && sj.chain) {
    if (sj.prec == 1) {
      if (sj.kw == 1)
        run_tile_chain<double, 1>(sj, smem, ctab, tile, ws);
      else
        run_tile_chain<double, 2>(sj, smem, ctab, tile, ws);
    } else {
      if (sj.kw == 1)
        run_tile_chain<float, 1>(sj, smem, ctab, tile, ws);
      else
        run_tile_chain<float, 2>(sj, smem, ctab, tile, ws);
    }
    return;
  }
  if (sj.prec == 1) {
    if (sj.kw == 1)
      run_tile<double, 1, SYS>(sj, smem, ctab, tile, ws);
    else
      run_tile<double, 2, SYS>(sj, smem, ctab, tile, ws);
  } else {
    if (sj.kw == 1)
      run_tile<float, 1, SYS>(sj, smem, ctab, tile, ws);
    else
      run_tile<float, 2, SYS>(sj, smem, ctab, tile, ws);
  }
}

// Each kernel holds some of the paths (see kernels.h); the host launches a job only in a kernel that
// holds its path (a bit-mask job may also run the general path: its columns and stream exist too).
// LAT: 0 = no lattice path; else the largest unrolled species count the kernel holds (2, 5 or 8);
// LATW: the words per cell set of its lattice jobs (1: up to 64 cells, 2: up to 128).
template <bool SYS, bool GENERAL, bool MASK, int LAT, int LATW>
__device__ __forceinline__ void dispatch_tile(const JobDesc& sj, uint8_t* smem, LevelSlot* ctab, const Tile& tile,
                                              WarpState& ws) {
  if constexpr (MASK) {
    if (sj.k2 == 1 || sj.k2 == 2) {
      dispatch_mask<SYS>(sj, smem, ctab, tile, ws);
      return;
    }
  }
  if constexpr (LAT > 0) {
    if (sj.lat && sj.lat_kmax <= static_cast<uint32_t>(LAT) && sj.lat_words == static_cast<uint32_t>(LATW)) {
      dispatch_lattice<SYS, LAT, LATW>(sj, smem, ctab, tile, ws);
      return;
    }
  }
  if constexpr (GENERAL) {
    if (!sj.lat || sj.trace) {  // a lattice job's shared memory holds the general layout only in traces
      dispatch_general<SYS>(sj, smem, ctab, tile, ws);
      return;
    }
  }
  // no path of this kernel fits the job: nothing is evaluated and the job is flagged
  if (threadIdx.x == 0) atomicMax(&sj.counters[kError], static_cast<unsigned long long>(kErrBadJob));
}

// Tiles are taken from q with one atomic per tile. A CTA stages a job's read-only data (cubes,
// windows, pair stream, packed species, masks) into shared memory with non-multicast bulk copies
// whenever its next tile belongs to another job. In live mode every tile ends with a level flush and
// a decrement of the job's tile count; the CTA that finishes a job's last tile publishes the job's
// generation in done[slot] (host-mapped memory).
template <bool GENERAL, bool MASK, int LAT, int LATW = 1>
__device__ __forceinline__ void engine_body(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles,
                                            uint32_t n_tiles, QueueCtl* q, const volatile int32_t* cancel,
                                            unsigned long long* status, volatile uint32_t* done) {
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ JobDesc sj;
  __shared__ LevelSlot ctab[kCtaLevelSlots];
  __shared__ unsigned long long s_tile;
  __shared__ uint32_t s_fail;
  __shared__ uint32_t s_counted;  // live mode: this CTA is counted in alive[its SM]
  __shared__ __align__(8) uint64_t s_bar;
  if (threadIdx.x == 0) {
    mbar_init(&s_bar, 1);
    s_fail = 0;
  }
  for (int i = threadIdx.x; i < kCtaLevelSlots; i += kBlock) ctab[i] = LevelSlot{0ull, 0ull, 0u, 0u};
  if constexpr (MASK)
    for (int i = threadIdx.x; i < kBlock / 32 * 96; i += kBlock) s_wacc[i] = 0u;
  const bool live = q->capacity != 0;
  int cur = -1;
  uint32_t cur_gen = 0;
  uint32_t phase = 0;
  WarpState ws;
  ws.big = nullptr;  // set with the first job
  if (threadIdx.x == 0) {
    s_counted = 0;
    if (live) {
      const uint32_t smid = sm_id();
      s_tile = kNoTile;
      if (owns_sm(q, smid)) {  // resident on one of its ring's SMs: counted while it stays
        if (q->alive && smid < q->n_owner) {
          atomicAdd(&q->alive[smid], 1u);
          s_counted = 1;
        }
        s_tile = claim_live(q, cancel, smid);
      }
    } else {
      s_tile = (cancel && *cancel) ? kNoTile : atomicAdd(&q->head, 1ull);
    }
  }
  for (;;) {
    __syncthreads();  // s_tile visible; every thread is done with the previous tile
    const unsigned long long ti = s_tile;
    if (ti == kNoTile || (!live && ti >= n_tiles)) break;
    // list mode: the next tile index is fetched now and only consumed after this tile
    unsigned long long next = kNoTile;
    if (!live && threadIdx.x == 0 && !(cancel && *cancel)) next = atomicAdd(&q->head, 1ull);
    Tile tile;
    {
      const uint4* src = reinterpret_cast<const uint4*>(&tiles[live ? ti % q->capacity : ti]);
      uint4* dst = reinterpret_cast<uint4*>(&tile);
      for (int k = 0; k < static_cast<int>(sizeof(Tile) / 16); ++k) dst[k] = __ldcg(src + k);
    }
    if (static_cast<int>(tile.job) != cur || tile.gen != cur_gen) {
      if (cur >= 0 && !live) flush_levels(ctab, sj);  // the previous job's levels leave first
      __syncthreads();
      const uint32_t* src = reinterpret_cast<const uint32_t*>(&jobs[tile.job]);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&sj);
      for (uint32_t i = threadIdx.x; i < sizeof(JobDesc) / 4; i += kBlock) dst[i] = __ldcg(src + i);
      __syncthreads();
      if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        uint32_t bytes = 0;
        for (uint32_t p = 0; p < sj.n_parts; ++p) bytes += sj.parts[p].static_bytes;
        mbar_expect_tx(&s_bar, bytes);
        if (!(sj.debug & kDebugSkipStaging))  // debug: nothing arrives, the wait below runs out
          for (uint32_t p = 0; p < sj.n_parts; ++p)
            bulk_copy_g2s(smem + sj.parts[p].smem_off, sj.blob + sj.parts[p].blob_off, sj.parts[p].static_bytes,
                          &s_bar);
      }
      if (!mbar_wait(&s_bar, phase, sj.wait_ns)) {
        atomicOr(&s_fail, 1u);
        // copies that were issued may still be landing in this CTA's shared memory: give them one
        // more bounded wait before the CTA leaves
        if (!(sj.debug & kDebugSkipStaging)) mbar_wait(&s_bar, phase, sj.wait_ns);
      }
      phase ^= 1u;
      __syncthreads();
      if (s_fail) {
        if (threadIdx.x == 0) {
          atomicMax(status, static_cast<unsigned long long>(kErrStageTimeout));
          atomicMax(&sj.counters[kError], static_cast<unsigned long long>(kErrStageTimeout));
        }
        break;
      }
      cur = static_cast<int>(tile.job);
      cur_gen = tile.gen;
      ws.reset(sj, smem);
    }
    if (sj.mode == 1)
      dispatch_tile<true, GENERAL, MASK, LAT, LATW>(sj, smem, ctab, tile, ws);
    else
      dispatch_tile<false, GENERAL, MASK, LAT, LATW>(sj, smem, ctab, tile, ws);
    __syncthreads();  // every thread is done with this tile before s_tile changes
    if (live) {
      flush_levels(ctab, sj);
      __threadfence();
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      atomicAdd(&sj.counters[kFinished], static_cast<unsigned long long>(sj.chain ? tile.chain_configs : tile.count));
      atomicAdd(&sj.counters[kTilesDone], 1ull);
      if (live) {
        __threadfence();  // this tile's counts land before the job's tile count drops
        if (atomicAdd(&sj.counters[kTilesLeft], ~0ull) == 1ull && done) {
          __threadfence_system();
          done[tile.job] = tile.gen;
        }
        s_tile = claim_live(q, cancel, sm_id());
      } else {
        s_tile = next;
      }
    }
  }
  if (cur >= 0 && !live) flush_levels(ctab, sj);
  if (live && threadIdx.x == 0) {
    if (s_counted) atomicAdd(&q->alive[sm_id()], ~0u);
    atomicAdd(&q->exited, 1u);
  }
}

}  // namespace sqsg
