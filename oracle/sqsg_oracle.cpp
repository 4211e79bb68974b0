// SQS optimisation oracle: a CPU restatement of the reference hot path.
//
// TEST INFRASTRUCTURE ONLY. This library is the checker for the GPU product and the timed
// "restated reference CPU path". Only tests/, __graft_entry__.smoke() and bench.py (its
// cpu_baseline leg and its --impl reference arm) may load it. The product package never links,
// imports or calls it.
//
// The reference (dgehringer/sqsgenerator 0.5.6) is header-only C++20 that cannot be compiled here:
// Eigen3, Boost.Multiprecision, Abseil and BS_thread_pool are absent. This file restates, in plain
// C++ with the same data types and the same floating-point operation order, the functions below.
// Every function cites the reference file:line it follows (paths relative to the reference root).
//
//   include/sqsgen/core/helpers/rapidhash.h:129-131,149-213  rapid_secret, rapid_mum, rapid_mix
//   include/sqsgen/core/shuffle.h:23-58                       rapidrand, random_bounded, shuffler
//   include/sqsgen/core/permutation.h:17-102                  num/rank/unrank/next permutation
//   include/sqsgen/core/optimization.h:74-103                 count_bonds, compute_objective
//   include/sqsgen/core/results.h:42-99                       sqs_result_collection
//   include/sqsgen/sqs.h:199-214,348-467                      optimizer worker loop + scheduling
//   BS_thread_pool v5 (bshoshany-thread-pool via vcpkg; version unpinned because the vcpkg
//   submodule is empty): detach_blocks splits [first, last) into num_blocks blocks of
//   total/num_blocks iterations, the first total%num_blocks blocks one larger; a pool with one
//   thread runs the blocks in submission order.
//
// Build: g++ -O2 -std=c++20 -ffp-contract=off -fPIC -shared (oracle/build.py). No -ffast-math and
// no FMA contraction, so double/float arithmetic rounds exactly like the reference's scalar code.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <shared_mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

extern "C" {

typedef struct {
  int32_t n_sites;
  int32_t n_species;
  int32_t n_shells;
  int32_t n_pairs;
  int32_t n_bounds;
  int32_t has_seed;
  const uint32_t* pairs;           // n_pairs * 3: (i, j, shell), i < j, shell in [0, n_shells)
  const uint8_t* species_packed;   // n_sites, packed species index in [0, n_species)
  const uint32_t* bounds;          // n_bounds * 2: shuffle windows [lo, hi)
  const void* prefactors;          // n_shells*n_species*n_species, row-major [s][a][b], prec type
  const void* pair_weights;        // already scaled by the shell weights
  const void* target;
  uint64_t seed;
} oracle_sublattice;

typedef struct {
  int32_t prec;                    // 0 = single (float), 1 = double
  int32_t iteration_mode;          // 0 = random, 1 = systematic
  int32_t sublattice_mode;         // 0 = interact, 1 = split
  int32_t n_sublattices;
  const oracle_sublattice* sublattices;
  uint64_t iterations;
  uint64_t chunk_size;
  uint64_t keep;
  int64_t max_results_per_objective;  // < 0: unset
  int32_t threads;
  int32_t share_seed_across_threads;  // 1: all threads race on one shuffler seed like the reference
} oracle_job;

typedef struct {
  uint64_t finished;
  uint64_t best_rank;
  double best_objective;
  double seconds;
} oracle_stats;
}

namespace oracle {

// ---------------------------------------------------------------------------------------------
// rapidhash (vendored MIT code in the reference): rapid_secret[0..1] core/helpers/rapidhash.h:129-131,
// rapid_mum (128-bit product, non-protected variant) :149-198, rapid_mix :209-213.
static constexpr uint64_t kSecret0 = 0x2d358dccaa6c78a5ull;
static constexpr uint64_t kSecret1 = 0x8bb84b93962eacc9ull;

static inline uint64_t rapid_mix(uint64_t a, uint64_t b) {
  __uint128_t r = static_cast<__uint128_t>(a) * b;
  return static_cast<uint64_t>(r) ^ static_cast<uint64_t>(r >> 64);
}

// core/shuffle.h:23-26. The seed lives behind a pointer so that several threads can share it the
// way the reference's shared shuffler does (relaxed loads/stores: the same machine code as the
// reference's unsynchronised member access, without undefined behaviour).
static inline uint64_t rapidrand(uint64_t* seed) {
  uint64_t s = __atomic_load_n(seed, __ATOMIC_RELAXED) + kSecret0;
  __atomic_store_n(seed, s, __ATOMIC_RELAXED);
  return rapid_mix(s, s ^ kSecret1);
}

// core/shuffle.h:28-32 — Lemire multiply-shift on the low 32 bits, no rejection.
static inline uint64_t random_bounded(uint64_t range, uint64_t* seed) {
  uint32_t x = static_cast<uint32_t>(rapidrand(seed));
  uint64_t m = static_cast<uint64_t>(x) * range;
  return m >> 32;
}

// core/shuffle.h:39-50 — Fisher-Yates per bound window, i from window size down to 2.
static void shuffle_random(uint8_t* c, const uint32_t* bounds, int n_bounds, uint64_t* seed) {
  for (int b = 0; b < n_bounds; ++b) {
    uint64_t lo = bounds[2 * b], hi = bounds[2 * b + 1];
    uint64_t w = hi - lo;
    for (uint64_t i = w; i > 1; i--) {
      uint64_t p = random_bounded(i, seed);
      std::swap(c[lo + i - 1], c[p + lo]);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// core/permutation.h. Ranks are boost::cpp_int in the reference; the parser rejects jobs whose
// permutation count exceeds uint64 (io/config/combined.h:88-95), so u64 ranks with 128-bit
// intermediates represent every rank the reference can iterate.
using u128 = __uint128_t;
static constexpr u128 kU64Max = std::numeric_limits<uint64_t>::max();

// core/permutation.h:17-32 — N! / prod(n_k!), evaluated as a product of binomials with overflow
// detection (the value is identical to the factorial quotient).
static bool num_permutations_counts(const std::vector<uint64_t>& hist, uint64_t* out) {
  u128 total = 1;
  uint64_t m = 0;
  for (uint64_t c : hist) {
    u128 binom = 1;
    for (uint64_t t = 1; t <= c; ++t) {
      binom = binom * (m + t) / t;
      if (binom > kU64Max) return false;
    }
    m += c;
    total *= binom;
    if (total > kU64Max) return false;
  }
  *out = static_cast<uint64_t>(total);
  return true;
}

static std::vector<uint64_t> histogram(const uint8_t* c, int n, int* num_species) {
  int k = 0;
  for (int i = 0; i < n; ++i) k = std::max(k, c[i] + 1);
  std::vector<uint64_t> h(k, 0);
  for (int i = 0; i < n; ++i) h[c[i]]++;
  if (num_species) *num_species = k;
  return h;
}

// core/permutation.h:34-50 (1-based rank over a configuration with dense values 0..K-1).
static uint64_t rank_permutation(const uint8_t* conf, int n) {
  int k = 0;
  for (int i = 0; i < n; ++i) k = std::max(k, conf[i] + 1);
  std::vector<uint64_t> hist(k, 0);
  u128 rank = 1, suffix = 1;
  for (int i = 0; i < n; i++) {
    int x = conf[(n - 1) - i];
    hist[x]++;
    for (int j = 0; j < x; j++) rank += suffix * hist[j] / hist[x];
    suffix = suffix * static_cast<u128>(i + 1) / hist[x];
  }
  return static_cast<uint64_t>(rank);
}

// core/permutation.h:52-78 (writes dense species indices 0..K-1 into conf).
static bool unrank_permutation(uint8_t* conf, int n, uint64_t to_rank) {
  int k = 0;
  std::vector<uint64_t> hist = histogram(conf, n, &k);
  // count() is an ordered map of the values present: drop absent values like the reference.
  std::vector<uint64_t> freqs;
  for (uint64_t h : hist)
    if (h) freqs.push_back(h);
  uint64_t total64;
  if (!num_permutations_counts(freqs, &total64)) return false;
  u128 total = total64, rank = to_rank;
  if (rank > total) return false;
  int pos = 0;
  int ns = static_cast<int>(freqs.size());
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < ns; j++) {
      u128 suffix_count = total * freqs[j] / static_cast<u128>(n - i);
      if (rank <= suffix_count) {
        conf[pos] = static_cast<uint8_t>(j);
        total = suffix_count;
        freqs[j]--;
        pos++;
        break;
      }
      rank -= suffix_count;
    }
  }
  return true;
}

// core/permutation.h:80-102 — lexicographic next permutation of a multiset.
static bool next_permutation(uint8_t* start, int64_t n) {
  if (n < 2) return false;
  int64_t l = n - 1, k = n - 2;
  while (start[k] >= start[k + 1]) {
    k -= 1;
    if (k < 0) return false;
  }
  while (start[k] >= start[l]) l -= 1;
  std::swap(start[k], start[l]);
  int64_t length = n - (k + 1);
  for (int64_t i = 0; i < length / 2; i++) std::swap(start[k + i + 1], start[n - i - 1]);
  return true;
}

// core/shuffle.h:69-88 — unrank inside the single window, remapping window values to dense
// indices when the window is not the whole configuration.
static bool unrank_window(uint8_t* conf, int n_sites, uint32_t lo, uint32_t hi, uint64_t rank) {
  if (lo == 0 && hi == static_cast<uint32_t>(n_sites)) return unrank_permutation(conf, n_sites, rank);
  int w = static_cast<int>(hi - lo);
  uint8_t present[256] = {0};
  for (int i = 0; i < w; ++i) present[conf[lo + i]] = 1;
  uint8_t fwd[256], rev[256];
  int k = 0;
  for (int v = 0; v < 256; ++v)
    if (present[v]) {
      fwd[v] = static_cast<uint8_t>(k);
      rev[k] = static_cast<uint8_t>(v);
      ++k;
    }
  std::vector<uint8_t> tmp(w);
  for (int i = 0; i < w; ++i) tmp[i] = fwd[conf[lo + i]];
  if (!unrank_permutation(tmp.data(), w, rank)) return false;
  for (int i = 0; i < w; ++i) conf[lo + i] = rev[tmp[i]];
  return true;
}

// ---------------------------------------------------------------------------------------------
// Per-sublattice data in the reference's own layouts: pairs as atom_pair<usize_t> (3 x u64,
// core/structure.h:21-27, usize_t = uint_fast32_t = u64 on x86-64 glibc), cubes as column-major
// Eigen::Tensor<T,3> (S,K,K) so element (s,a,b) sits at s + S*(a + K*b) (types.h:37).
struct Pair {
  uint64_t i, j, shell;
};

template <class T> struct Sublattice {
  int n_sites = 0, K = 0, S = 0;
  std::vector<Pair> pairs;
  std::vector<uint8_t> species_packed;
  std::vector<uint32_t> bounds;
  std::vector<T> f, w, t;  // column-major cubes
  uint64_t seed = 0;
  bool has_seed = false;

  size_t cidx(int s, int a, int b) const { return s + static_cast<size_t>(S) * (a + static_cast<size_t>(K) * b); }

  void load(const oracle_sublattice& d) {
    n_sites = d.n_sites;
    K = d.n_species;
    S = d.n_shells;
    pairs.resize(d.n_pairs);
    for (int p = 0; p < d.n_pairs; ++p)
      pairs[p] = Pair{d.pairs[3 * p], d.pairs[3 * p + 1], d.pairs[3 * p + 2]};
    species_packed.assign(d.species_packed, d.species_packed + d.n_sites);
    bounds.assign(d.bounds, d.bounds + 2 * d.n_bounds);
    size_t cube = static_cast<size_t>(S) * K * K;
    f.resize(cube);
    w.resize(cube);
    t.resize(cube);
    const T* fp = static_cast<const T*>(d.prefactors);
    const T* wp = static_cast<const T*>(d.pair_weights);
    const T* tp = static_cast<const T*>(d.target);
    for (int s = 0; s < S; ++s)
      for (int a = 0; a < K; ++a)
        for (int b = 0; b < K; ++b) {
          size_t rm = (static_cast<size_t>(s) * K + a) * K + b;
          f[cidx(s, a, b)] = fp[rm];
          w[cidx(s, a, b)] = wp[rm];
          t[cidx(s, a, b)] = tp[rm];
        }
    seed = d.seed;
    has_seed = d.has_seed != 0;
  }
};

// core/optimization.h:74-77 — ordered counts bonds(s, species[i], species[j]) over i<j pairs.
static inline void count_bonds(std::vector<uint64_t>& bonds, const std::vector<Pair>& pairs,
                               const uint8_t* species, int S, int K) {
  std::fill(bonds.begin(), bonds.end(), 0);
  for (const Pair& p : pairs)
    bonds[p.shell + static_cast<size_t>(S) * (species[p.i] + static_cast<size_t>(K) * species[p.j])]++;
}

// core/helpers/numeric.h:16
template <class T> static inline T absolute(T a) { return a > 0 ? a : -a; }

// core/optimization.h:79-103 — same loop order and accumulation in T.
template <class T>
static inline T compute_objective(std::vector<T>& sro, const std::vector<uint64_t>& bonds,
                                  const Sublattice<T>& sl) {
  const int S = sl.S, K = sl.K;
  std::fill(sro.begin(), sro.end(), T(0.0));
  T objective{0.0};
  for (int s = 0; s < S; ++s)
    for (int xi = 0; xi < K; ++xi) {
      T sigma_xx = T(1.0) - static_cast<T>(bonds[sl.cidx(s, xi, xi)]) * sl.f[sl.cidx(s, xi, xi)];
      sro[sl.cidx(s, xi, xi)] = sigma_xx;
      objective += sl.w[sl.cidx(s, xi, xi)] * absolute(sigma_xx - sl.t[sl.cidx(s, xi, xi)]);
      for (int eta = xi + 1; eta < K; ++eta) {
        uint64_t pair_bonds = bonds[sl.cidx(s, xi, eta)] + bonds[sl.cidx(s, eta, xi)];
        T sigma = T(1.0) - static_cast<T>(pair_bonds) * sl.f[sl.cidx(s, xi, eta)];
        sro[sl.cidx(s, xi, eta)] = sigma;
        sro[sl.cidx(s, eta, xi)] = sigma;
        objective += sl.w[sl.cidx(s, xi, eta)] * absolute(sigma - sl.t[sl.cidx(s, xi, eta)]);
      }
    }
  return objective;
}

// ---------------------------------------------------------------------------------------------
// core/results.h:42-99 — results keyed by exact objective, deduplicated by configuration; a
// sorted vector of distinct objectives gives nth_best(). Never evicts.
template <class T> struct Result {
  T objective;
  std::vector<T> sub_objectives;          // one per sublattice
  std::vector<uint8_t> species;           // concatenated per sublattice (packed, sorted order)
  std::vector<T> sro;                     // concatenated column-major cubes
};

template <class T> class ResultCollection {
 public:
  void insert(Result<T>&& r) {
    std::unique_lock lock(mutex_);
    auto it = data_.find(r.objective);
    if (it != data_.end()) {
      it->second.emplace(r.species, std::move(r));
      return;
    }
    T obj = r.objective;
    std::map<std::vector<uint8_t>, Result<T>> set;
    set.emplace(r.species, std::move(r));
    data_.emplace(obj, std::move(set));
    auto pos = std::lower_bound(objectives_.begin(), objectives_.end(), obj);
    if (pos == objectives_.end() || obj < *pos) objectives_.insert(pos, obj);
  }
  size_t results_for_objective(T objective) {
    std::shared_lock lock(mutex_);
    auto it = data_.find(objective);
    return it == data_.end() ? 0 : it->second.size();
  }
  T nth_best(size_t n) {
    std::shared_lock lock(mutex_);
    if (n >= objectives_.size()) return std::numeric_limits<T>::infinity();
    return objectives_[n];
  }
  // Sorted by objective, then by configuration (the reference's hash-set order is arbitrary).
  std::vector<Result<T>> flatten() {
    std::vector<Result<T>> out;
    for (auto& [obj, set] : data_)
      for (auto& [sp, r] : set) out.push_back(r);
    return out;
  }

 private:
  std::shared_mutex mutex_;
  std::vector<T> objectives_;
  std::map<T, std::map<std::vector<uint8_t>, Result<T>>> data_;
};

template <class T> struct Output {
  std::vector<Result<T>> results;
  oracle_stats stats{};
  std::vector<int> n_sites, S, K;
};

// sqs.h:199-214 atomics + sqs.h:299-467 optimizer::run for one rank (no MPI).
template <class T> static Output<T>* optimize(const oracle_job& job) {
  const bool split = job.sublattice_mode == 1;
  const bool systematic = job.iteration_mode == 1;
  const int nsl = job.n_sublattices;
  std::vector<Sublattice<T>> sls(nsl);
  for (int i = 0; i < nsl; ++i) sls[i].load(job.sublattices[i]);
  if (systematic && (split || nsl != 1 || sls[0].bounds.size() != 2))
    throw std::invalid_argument("systematic mode needs one sublattice with one window");

  // One shuffler per sublattice (optimization_config.h:91). Seeds are shared by all threads.
  std::vector<uint64_t> seeds(nsl);
  for (int i = 0; i < nsl; ++i) seeds[i] = sls[i].seed;

  std::atomic<T> best_objective{std::numeric_limits<T>::max()};
  std::atomic<T> search_objective{std::numeric_limits<T>::max()};
  std::atomic<uint64_t> finished{0}, best_rank{0};
  std::atomic<T> stat_best{std::numeric_limits<T>::infinity()};
  std::mutex stat_mutex;
  ResultCollection<T> results;
  const uint64_t keep = job.keep;
  const bool cap = job.max_results_per_objective >= 0;
  const uint64_t cap_value = cap ? static_cast<uint64_t>(job.max_results_per_objective) : 0;

  // BS_thread_pool v5 blocks(): num_blocks = (end - start) / chunk_size (sqs.h:461-466).
  const uint64_t first = 0, last = job.iterations;
  uint64_t total = last - first;
  uint64_t nb = job.chunk_size ? total / job.chunk_size : 0;
  if (nb == 0) nb = static_cast<uint64_t>(std::max(1, job.threads));
  uint64_t block_size = 0, remainder = 0;
  if (total > 0) {
    nb = std::min(nb, total);
    block_size = total / nb;
    remainder = total % nb;
    if (block_size == 0) {
      block_size = 1;
      nb = total > 1 ? total : 1;
    }
  } else {
    nb = 0;
  }
  auto block_start = [&](uint64_t b) { return first + b * block_size + std::min(b, remainder); };
  auto block_end = [&](uint64_t b) { return b == nb - 1 ? last : block_start(b + 1); };

  std::atomic<uint64_t> next_block{0};
  auto worker = [&](std::vector<uint64_t>* private_seeds) {
    uint64_t* seed_ptr = private_seeds ? private_seeds->data() : seeds.data();
    std::vector<std::vector<uint64_t>> bonds(nsl);
    std::vector<std::vector<T>> sro(nsl);
    for (int s = 0; s < nsl; ++s) {
      bonds[s].assign(static_cast<size_t>(sls[s].S) * sls[s].K * sls[s].K, 0);
      sro[s].assign(bonds[s].size(), T(0));
    }
    std::vector<T> objective(nsl, T(0));
    std::vector<std::vector<uint8_t>> species(nsl);
    while (true) {
      uint64_t b = next_block.fetch_add(1);
      if (b >= nb) break;
      uint64_t rstart = block_start(b), rend = block_end(b);
      for (int s = 0; s < nsl; ++s) species[s] = sls[s].species_packed;  // sqs.h:374
      if (systematic) {                                                   // sqs.h:377-378
        if (!unrank_window(species[0].data(), sls[0].n_sites, sls[0].bounds[0], sls[0].bounds[1],
                           rstart + 1))
          throw std::out_of_range("rank larger than the number of permutations");
      }
      for (uint64_t i = rstart; i < rend; ++i) {
        if (!split) {
          count_bonds(bonds[0], sls[0].pairs, species[0].data(), sls[0].S, sls[0].K);  // sqs.h:400
          objective[0] = compute_objective(sro[0], bonds[0], sls[0]);              // sqs.h:401
        } else {
          for (int s = 0; s < nsl; ++s) {                                          // sqs.h:404-413
            shuffle_random(species[s].data(), sls[s].bounds.data(),
                           static_cast<int>(sls[s].bounds.size() / 2), &seed_ptr[s]);
            count_bonds(bonds[s], sls[s].pairs, species[s].data(), sls[s].S, sls[s].K);
            objective[s] = compute_objective(sro[s], bonds[s], sls[s]);
          }
        }
        T value;
        if (!split) {
          value = objective[0];
        } else {  // core/helpers/fold.h:51-53: left fold from T(0)
          value = T(0);
          for (int s = 0; s < nsl; ++s) value = value + objective[s];
        }
        if (value <= search_objective.load()) {                                    // sqs.h:421
          if (cap && results.results_for_objective(value) > cap_value) continue;   // sqs.h:423-426
          Result<T> r;
          r.objective = value;
          r.sub_objectives = objective;
          for (int s = 0; s < nsl; ++s) {
            r.species.insert(r.species.end(), species[s].begin(), species[s].end());
            r.sro.insert(r.sro.end(), sro[s].begin(), sro[s].end());
          }
          results.insert(std::move(r));                                            // sqs.h:432
          T nth = results.nth_best(keep);                                          // sqs.h:435
          if (value < best_objective.load()) best_objective.store(value);
          if (nth < search_objective.load()) search_objective.store(nth);
          {                                                                        // sqs.h:437
            std::scoped_lock l(stat_mutex);
            if (value < stat_best.load()) {
              stat_best.store(value);
              best_rank.store(rstart + i);
            }
          }
        }
        if (!split) {                                                              // sqs.h:439-440
          if (systematic)
            next_permutation(species[0].data() + sls[0].bounds[0],
                             static_cast<int64_t>(sls[0].bounds[1] - sls[0].bounds[0]));
          else
            shuffle_random(species[0].data(), sls[0].bounds.data(),
                           static_cast<int>(sls[0].bounds.size() / 2), &seed_ptr[0]);
        }
      }
      finished.fetch_add(rend - rstart);
    }
  };

  int nt = std::max(1, job.threads);
  auto t0 = std::chrono::steady_clock::now();
  if (nt == 1) {
    worker(nullptr);
  } else {
    std::vector<std::thread> pool;
    std::vector<std::vector<uint64_t>> private_seeds(nt);
    for (int t = 0; t < nt; ++t) {
      private_seeds[t] = seeds;
      for (auto& s : private_seeds[t]) s += 0x9e3779b97f4a7c15ull * static_cast<uint64_t>(t + 1);
      pool.emplace_back(worker, job.share_seed_across_threads ? nullptr : &private_seeds[t]);
    }
    for (auto& th : pool) th.join();
  }
  auto t1 = std::chrono::steady_clock::now();

  auto* out = new Output<T>();
  out->results = results.flatten();
  out->stats.finished = finished.load();
  out->stats.best_rank = best_rank.load();
  out->stats.best_objective = static_cast<double>(stat_best.load());
  out->stats.seconds = std::chrono::duration<double>(t1 - t0).count();
  for (auto& s : sls) {
    out->n_sites.push_back(s.n_sites);
    out->S.push_back(s.S);
    out->K.push_back(s.K);
  }
  return out;
}

// Copies result `index`: total objective, per-sublattice objectives, concatenated packed species,
// concatenated row-major sro cubes. Values are written in the job's precision.
template <class T>
static void copy_result(Output<T>* o, uint64_t index, void* objective, void* sub_objectives,
                        uint8_t* species, void* sro) {
  const Result<T>& r = o->results[index];
  *static_cast<T*>(objective) = r.objective;
  std::memcpy(sub_objectives, r.sub_objectives.data(), sizeof(T) * r.sub_objectives.size());
  std::memcpy(species, r.species.data(), r.species.size());
  size_t off = 0, rm_off = 0;
  T* out = static_cast<T*>(sro);
  for (size_t s = 0; s < o->S.size(); ++s) {
    int S = o->S[s], K = o->K[s];
    for (int a = 0; a < S; ++a)
      for (int x = 0; x < K; ++x)
        for (int y = 0; y < K; ++y)
          out[rm_off + (static_cast<size_t>(a) * K + x) * K + y] =
              r.sro[off + a + static_cast<size_t>(S) * (x + static_cast<size_t>(K) * y)];
    off += static_cast<size_t>(S) * K * K;
    rm_off += static_cast<size_t>(S) * K * K;
  }
}

// Exhaustive enumeration of one window (core/permutation.h + core/optimization.h restated above),
// keeping per distinct objective the number of configurations and two order-independent 32-bit sums
// of splitmix64(rank). Used to compare result sets too large to materialise. Every thread keeps only
// its keep+1 smallest distinct objectives: a value beyond a thread's (keep+1)-th smallest cannot be
// among the (keep+1) smallest overall.
static inline uint64_t splitmix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

struct LevelAcc {
  uint64_t count = 0;
  uint32_t sa = 0, sb = 0;
};

template <class T>
static std::map<T, LevelAcc> systematic_levels(const oracle_sublattice& d, int threads, uint64_t keep,
                                               uint64_t first, uint64_t count) {
  Sublattice<T> sl;
  sl.load(d);
  const uint32_t lo = sl.bounds[0], hi = sl.bounds[1];
  std::vector<uint8_t> win(sl.species_packed.begin() + lo, sl.species_packed.begin() + hi);
  uint64_t total;
  {
    std::vector<uint64_t> h = histogram(win.data(), static_cast<int>(win.size()), nullptr), f;
    for (uint64_t x : h)
      if (x) f.push_back(x);
    if (!num_permutations_counts(f, &total)) throw std::out_of_range("too many permutations");
  }
  if (first > total) throw std::out_of_range("first rank beyond the permutation count");
  const uint64_t span = count ? std::min(count, total - first) : total - first;
  const int nt = std::max(1, threads);
  const uint64_t nblocks = std::max<uint64_t>(1, std::min<uint64_t>(span, static_cast<uint64_t>(nt) * 64));
  std::atomic<uint64_t> next{0};
  std::vector<std::map<T, LevelAcc>> per(nt);
  auto work = [&](int tid) {
    std::vector<uint64_t> bonds(static_cast<size_t>(sl.S) * sl.K * sl.K);
    std::vector<T> sro(bonds.size());
    std::map<T, LevelAcc>& m = per[tid];
    while (true) {
      uint64_t b = next.fetch_add(1);
      if (b >= nblocks) break;
      uint64_t r0 = 1 + first + span / nblocks * b + std::min(b, span % nblocks);
      uint64_t r1 = 1 + first + span / nblocks * (b + 1) + std::min(b + 1, span % nblocks);
      std::vector<uint8_t> sp = sl.species_packed;
      unrank_window(sp.data(), sl.n_sites, lo, hi, r0);
      for (uint64_t r = r0; r < r1; ++r) {
        count_bonds(bonds, sl.pairs, sp.data(), sl.S, sl.K);
        T o = compute_objective(sro, bonds, sl);
        if (m.size() <= keep || o <= std::prev(m.end())->first) {
          LevelAcc& a = m[o];
          uint64_t h = splitmix64(r);
          a.count++;
          a.sa += static_cast<uint32_t>(h);
          a.sb += static_cast<uint32_t>(h >> 32);
          if (m.size() > keep + 1) m.erase(std::prev(m.end()));
        }
        next_permutation(sp.data() + lo, static_cast<int64_t>(hi - lo));
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t) pool.emplace_back(work, t);
  for (auto& th : pool) th.join();
  std::map<T, LevelAcc> all;
  for (auto& m : per)
    for (auto& [v, a] : m) {
      LevelAcc& x = all[v];
      x.count += a.count;
      x.sa += a.sa;
      x.sb += a.sb;
    }
  while (all.size() > keep + 1) all.erase(std::prev(all.end()));
  return all;
}

// count_bonds + compute_objective for n configurations (species n x N): ordered bonds row-major
// (n x S*K*K) and objectives (n values of the job's precision).
template <class T>
static void evaluate_many(const oracle_sublattice* d, uint64_t n, const uint8_t* species, uint64_t* bonds_rm, T* obj) {
  Sublattice<T> sl;
  sl.load(*d);
  const size_t skk = static_cast<size_t>(sl.S) * sl.K * sl.K;
  std::vector<uint64_t> b(skk);
  std::vector<T> sro(skk);
  for (uint64_t k = 0; k < n; ++k) {
    const uint8_t* sp = species + k * sl.n_sites;
    count_bonds(b, sl.pairs, sp, sl.S, sl.K);
    obj[k] = compute_objective(sro, b, sl);
    for (int s = 0; s < sl.S; ++s)
      for (int a = 0; a < sl.K; ++a)
        for (int c = 0; c < sl.K; ++c) bonds_rm[k * skk + (static_cast<size_t>(s) * sl.K + a) * sl.K + c] = b[sl.cidx(s, a, c)];
  }
}

struct Handle {
  int prec;
  void* out;
  std::string error;
};

thread_local std::string g_error;

}  // namespace oracle

using namespace oracle;

extern "C" {

const char* oracle_last_error() { return g_error.c_str(); }

uint64_t oracle_rapidrand(uint64_t* seed) { return rapidrand(seed); }

uint64_t oracle_random_bounded(uint64_t range, uint64_t* seed) { return random_bounded(range, seed); }

void oracle_shuffle_random(uint8_t* conf, const uint32_t* bounds, int n_bounds, uint64_t* seed) {
  shuffle_random(conf, bounds, n_bounds, seed);
}

// Returns 1 on success, 0 if the count does not fit in 64 bits.
int oracle_num_permutations(const uint8_t* conf, int n, uint64_t* out) {
  std::vector<uint64_t> h = histogram(conf, n, nullptr), f;
  for (uint64_t x : h)
    if (x) f.push_back(x);
  return num_permutations_counts(f, out) ? 1 : 0;
}

uint64_t oracle_rank_permutation(const uint8_t* conf, int n) { return rank_permutation(conf, n); }

int oracle_unrank_permutation(uint8_t* conf, int n, uint64_t rank) {
  return unrank_permutation(conf, n, rank) ? 1 : 0;
}

int oracle_next_permutation(uint8_t* conf, int n) { return next_permutation(conf, n) ? 1 : 0; }

// Ordered bond counts like core/optimization.h:74-77, returned row-major [s][a][b].
void oracle_count_bonds(const oracle_sublattice* d, const uint8_t* species, uint64_t* bonds_rm) {
  Sublattice<double> sl;
  sl.n_sites = d->n_sites;
  sl.K = d->n_species;
  sl.S = d->n_shells;
  sl.pairs.resize(d->n_pairs);
  for (int p = 0; p < d->n_pairs; ++p)
    sl.pairs[p] = Pair{d->pairs[3 * p], d->pairs[3 * p + 1], d->pairs[3 * p + 2]};
  std::vector<uint64_t> b(static_cast<size_t>(sl.S) * sl.K * sl.K);
  count_bonds(b, sl.pairs, species, sl.S, sl.K);
  for (int s = 0; s < sl.S; ++s)
    for (int a = 0; a < sl.K; ++a)
      for (int c = 0; c < sl.K; ++c) bonds_rm[(static_cast<size_t>(s) * sl.K + a) * sl.K + c] = b[sl.cidx(s, a, c)];
}

// count_bonds + compute_objective for one configuration; sro returned row-major.
double oracle_evaluate_d(const oracle_sublattice* d, const uint8_t* species, double* sro_rm) {
  Sublattice<double> sl;
  sl.load(*d);
  std::vector<uint64_t> b(static_cast<size_t>(sl.S) * sl.K * sl.K);
  std::vector<double> sro(b.size());
  count_bonds(b, sl.pairs, species, sl.S, sl.K);
  double o = compute_objective(sro, b, sl);
  for (int s = 0; s < sl.S; ++s)
    for (int a = 0; a < sl.K; ++a)
      for (int c = 0; c < sl.K; ++c) sro_rm[(static_cast<size_t>(s) * sl.K + a) * sl.K + c] = sro[sl.cidx(s, a, c)];
  return o;
}

float oracle_evaluate_f(const oracle_sublattice* d, const uint8_t* species, float* sro_rm) {
  Sublattice<float> sl;
  sl.load(*d);
  std::vector<uint64_t> b(static_cast<size_t>(sl.S) * sl.K * sl.K);
  std::vector<float> sro(b.size());
  count_bonds(b, sl.pairs, species, sl.S, sl.K);
  float o = compute_objective(sro, b, sl);
  for (int s = 0; s < sl.S; ++s)
    for (int a = 0; a < sl.K; ++a)
      for (int c = 0; c < sl.K; ++c) sro_rm[(static_cast<size_t>(s) * sl.K + a) * sl.K + c] = sro[sl.cidx(s, a, c)];
  return o;
}

void oracle_evaluate_many(const oracle_sublattice* d, int prec, uint64_t n, const uint8_t* species, uint64_t* bonds,
                          void* obj) {
  if (prec == 1)
    evaluate_many<double>(d, n, species, bonds, static_cast<double*>(obj));
  else
    evaluate_many<float>(d, n, species, bonds, static_cast<float*>(obj));
}

void* oracle_optimize(const oracle_job* job) {
  try {
    auto* h = new Handle{job->prec, nullptr, ""};
    if (job->prec == 1)
      h->out = optimize<double>(*job);
    else
      h->out = optimize<float>(*job);
    return h;
  } catch (std::exception const& e) {
    g_error = e.what();
    return nullptr;
  }
}

void oracle_result_free(void* hp) {
  auto* h = static_cast<Handle*>(hp);
  if (!h) return;
  if (h->prec == 1)
    delete static_cast<Output<double>*>(h->out);
  else
    delete static_cast<Output<float>*>(h->out);
  delete h;
}

uint64_t oracle_result_count(void* hp) {
  auto* h = static_cast<Handle*>(hp);
  return h->prec == 1 ? static_cast<Output<double>*>(h->out)->results.size()
                      : static_cast<Output<float>*>(h->out)->results.size();
}

void oracle_result_stats(void* hp, oracle_stats* st) {
  auto* h = static_cast<Handle*>(hp);
  *st = h->prec == 1 ? static_cast<Output<double>*>(h->out)->stats
                     : static_cast<Output<float>*>(h->out)->stats;
}

// core/optimization.h:35-72 — sites sorted by sublattice index with std::sort (libstdc++, not
// stable) and the same comparator, then the windows cut between sublattices. Returns the window
// count (windows holds up to 2 * cap entries).
int oracle_sort_by_sublattice(const uint32_t* sl_of_site, int n, int n_sublattices, uint32_t* order,
                              uint32_t* windows, int cap) {
  struct Site {
    uint64_t index;
    uint64_t pad[4];  // sites are moved as whole objects in the reference; layout does not matter
  };
  std::vector<Site> sites(n);
  for (int i = 0; i < n; ++i) sites[i].index = static_cast<uint64_t>(i);
  std::sort(sites.begin(), sites.end(),
            [&](const Site& a, const Site& b) { return sl_of_site[a.index] < sl_of_site[b.index]; });
  std::vector<uint32_t> idx(n);
  for (int i = 0; i < n; ++i) {
    order[i] = static_cast<uint32_t>(sites[i].index);
    idx[i] = sl_of_site[sites[i].index];
  }
  int count = 0, lower = 0;
  auto push = [&](int lo, int hi) {
    if (count < cap) {
      windows[2 * count] = static_cast<uint32_t>(lo);
      windows[2 * count + 1] = static_cast<uint32_t>(hi);
    }
    ++count;
  };
  for (int i = 0; i < n; ++i) {
    if (idx[i] != idx[lower]) {
      push(lower, i);
      lower = i;
      if (idx[i] == static_cast<uint32_t>(n_sublattices)) break;
    } else if (i == n - 1) {
      push(lower, i + 1);
    }
  }
  return count;
}

// Writes up to *n levels (value as double, count, checksum = sa | sb << 32); returns the count.
int oracle_systematic_levels(const oracle_sublattice* d, int prec, int threads, uint64_t keep, uint64_t first,
                             uint64_t count, double* values, uint64_t* counts, uint64_t* checksums, int cap) {
  try {
    int k = 0;
    auto emit = [&](auto const& m) {
      for (auto& [v, a] : m) {
        if (k >= cap) break;
        values[k] = static_cast<double>(v);
        counts[k] = a.count;
        checksums[k] = static_cast<uint64_t>(a.sa) | (static_cast<uint64_t>(a.sb) << 32);
        ++k;
      }
    };
    if (prec == 1)
      emit(systematic_levels<double>(*d, threads, keep, first, count));
    else
      emit(systematic_levels<float>(*d, threads, keep, first, count));
    return k;
  } catch (std::exception const& e) {
    g_error = e.what();
    return -1;
  }
}

void oracle_result_get(void* hp, uint64_t index, void* objective, void* sub_objectives,
                       uint8_t* species, void* sro) {
  auto* h = static_cast<Handle*>(hp);
  if (h->prec == 1)
    copy_result(static_cast<Output<double>*>(h->out), index, objective, sub_objectives, species, sro);
  else
    copy_result(static_cast<Output<float>*>(h->out), index, objective, sub_objectives, species, sro);
}
}
