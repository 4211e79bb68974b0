// Host-side job preparation: validates a job and lays out what the device engine reads — the job
// descriptor (part offsets, paths, record layout) and the job blob (per part: objective cubes,
// windows, packed species, path-specific tables and the grouped pair stream) — and cuts the job's
// configuration range into tiles. Shared by sqsg_optimize, the batched and served forms, the launch
// plan and the allocation-free entry point, so that every entry point evaluates the same job the
// same way.
//
// Restates the per-sublattice data of optimization_config::from_config
// (include/sqsgen/core/optimization_config.h:59-141) in the engine's layout.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "permutation.h"
#include "prepare.h"
#include "sqsg_internal.h"
#include "tiles.h"

namespace sqsg {


template <class T> static void copy_cube(std::vector<uint8_t>& blob, size_t off, const void* src, size_t n) {
  std::memcpy(blob.data() + off, src, n * sizeof(T));
}

// Pair stream of a part: for each shell s and site i (ascending) a header word (s | cnt << 8), the
// byte offset of i in a species column, and cnt byte offsets of its neighbours j > i in shell s.
// The grouped pair stream of one part: for each (shell s, site i) the sites j > i of its pairs, in
// groups of at most kMaxGroup. Narrow form (every column offset below 2^16, i.e. N <= 512): one
// header word  ioff | s << 16 | cnt << 24  and the cnt column offsets as 16-bit halves, two per
// word. Wide form: header words  s | cnt << 8  and  ioff, then one word per offset.
static bool narrow_stream(uint32_t n_sites) { return host_site_off(n_sites ? n_sites - 1 : 0) < 0x10000u; }

// CTAs of the general-path kernel (sqsg_engine_wide, at most kMinBlocksWide) that fit on one SM of
// `device` with `dynamic_smem` bytes each, from the device's shared memory per SM and per-block
// reservation and the kernel's static shared memory (an estimate that needs no CUDA context).
int ctas_per_sm(int device, size_t dynamic_smem) {
  static std::mutex m;
  static std::map<int, std::pair<size_t, size_t>> cache;  // device -> (smem per SM, reserved per block)
  std::pair<size_t, size_t> dev{233472, 1024};
  {
    std::lock_guard<std::mutex> l(m);
    auto it = cache.find(device);
    if (it != cache.end()) {
      dev = it->second;
    } else {
      int per_sm = 0, reserved = 0;
      if (cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device) == cudaSuccess &&
          cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device) == cudaSuccess)
        dev = {static_cast<size_t>(per_sm), static_cast<size_t>(reserved)};
      else
        cudaGetLastError();
      cache[device] = dev;
    }
  }
  const size_t static_smem = sizeof(JobDesc) + kCtaLevelSlots * sizeof(LevelSlot) + 128;
  const size_t per_cta = align_up(dynamic_smem + static_smem, 128) + dev.second;
  return static_cast<int>(std::min<size_t>(kMinBlocksWide, dev.first / per_cta));
}

static std::vector<uint32_t> build_stream(const sqsg_sublattice& sl) {
  const uint32_t N = sl.n_sites, S = sl.n_shells, P = sl.n_pairs;
  std::vector<std::vector<uint32_t>> by(static_cast<size_t>(S) * N);
  std::vector<uint64_t> per_shell(S, 0);
  for (uint32_t p = 0; p < P; ++p) {
    uint32_t i = sl.pairs[3 * p], j = sl.pairs[3 * p + 1], s = sl.pairs[3 * p + 2];
    if (i >= N || j >= N) throw std::out_of_range("pair index out of range");
    if (s >= S) throw std::out_of_range("pair shell index out of range");
    if (i == j) throw std::invalid_argument("pair with i == j");
    if (i > j) std::swap(i, j);  // ordered counts are defined for i < j (structure.h:445-447)
    by[static_cast<size_t>(s) * N + i].push_back(j);
    per_shell[s]++;
  }
  for (uint32_t s = 0; s < S; ++s)
    if (per_shell[s] > 0xffffu)
      throw unsupported_error("a shell holds more than 65535 pairs; the 16-bit bond counters cannot hold it");
  const bool narrow = narrow_stream(N);
  std::vector<uint32_t> st;
  st.reserve(P + 2 * static_cast<size_t>(S) * N);
  for (uint32_t s = 0; s < S; ++s)
    for (uint32_t i = 0; i < N; ++i) {
      auto& js = by[static_cast<size_t>(s) * N + i];
      std::sort(js.begin(), js.end());
      for (size_t b = 0; b < js.size(); b += kMaxGroup) {
        uint32_t cnt = static_cast<uint32_t>(std::min<size_t>(kMaxGroup, js.size() - b));
        if (narrow) {
          st.push_back(host_site_off(i) | (s << 16) | (cnt << 24));
          for (uint32_t e = 0; e < cnt; e += 2) {
            const uint32_t lo = host_site_off(js[b + e]);
            const uint32_t hi = e + 1 < cnt ? host_site_off(js[b + e + 1]) : 0u;
            st.push_back(lo | (hi << 16));
          }
        } else {
          st.push_back(s | (cnt << 8));
          st.push_back(host_site_off(i));
          for (uint32_t e = 0; e < cnt; ++e) st.push_back(host_site_off(js[b + e]));
        }
      }
    }
  return st;
}

static uint64_t window_permutations(const sqsg_sublattice& sl, PartDesc& pd) {
  const uint32_t lo = sl.windows[0], hi = sl.windows[1];
  uint32_t counts[256] = {0};
  for (uint32_t x = lo; x < hi; ++x) counts[sl.species[x]]++;
  uint32_t k = 0;
  uint32_t dense[kMaxSpecies];
  for (uint32_t v = 0; v < 256; ++v)
    if (counts[v]) {
      if (k >= kMaxSpecies) throw unsupported_error("more than 8 species in the systematic window");
      pd.unrank_rev[k] = static_cast<uint8_t>(v);
      pd.unrank_hist[k] = counts[v];
      dense[k] = counts[v];
      ++k;
    }
  pd.unrank_k = k;
  uint64_t total = 0;
  if (!num_permutations_counts(dense, static_cast<int>(k), &total))
    throw std::out_of_range("The number of permutations to test does not fit in 64 bits");
  return total;
}

PreparedJob prepare(const sqsg_job& job, uint64_t trace_capacity) {
  PreparedJob pj;
  if (job.prec != SQSG_PREC_SINGLE && job.prec != SQSG_PREC_DOUBLE) throw std::invalid_argument("invalid prec");
  if (job.iteration_mode != SQSG_ITERATION_RANDOM && job.iteration_mode != SQSG_ITERATION_SYSTEMATIC)
    throw std::invalid_argument("invalid iteration mode");
  if (job.sublattice_mode != SQSG_SUBLATTICE_INTERACT && job.sublattice_mode != SQSG_SUBLATTICE_SPLIT)
    throw std::invalid_argument("invalid sublattice mode");
  if (!job.sublattices || job.n_sublattices == 0) throw std::invalid_argument("no sublattices");
  if (job.sublattice_mode == SQSG_SUBLATTICE_INTERACT && job.n_sublattices != 1)
    throw std::invalid_argument("interact mode takes one optimised structure (windows carry the sublattices)");
  if (job.n_sublattices > static_cast<uint32_t>(kMaxParts))
    throw unsupported_error("more than 8 sublattices in split mode");
  if (job.iteration_mode == SQSG_ITERATION_SYSTEMATIC && job.sublattice_mode == SQSG_SUBLATTICE_SPLIT)
    throw std::invalid_argument(
        "It is not possible to do an exhaustive search on multiple sublattices in mode \"split\"");
  if (job.keep == 0) throw std::invalid_argument("The number of best kept structures must be greater than 0");
  if (job.keep > static_cast<uint64_t>(kMaxKeep))
    throw unsupported_error("keep > " + std::to_string(kMaxKeep) + " is not supported (the warps' best lists)");
  pj.prec = job.prec;
  pj.tsz = job.prec == SQSG_PREC_DOUBLE ? 8 : 4;
  pj.systematic = job.iteration_mode == SQSG_ITERATION_SYSTEMATIC;
  pj.keep = job.keep;
  pj.max_rpo = job.max_results_per_objective;
  pj.max_results = job.max_results;
  JobDesc& d = pj.desc;
  d.prec = static_cast<uint32_t>(job.prec);
  d.mode = pj.systematic ? 1 : 0;
  d.n_parts = job.n_sublattices;
  d.keep = static_cast<uint32_t>(job.keep);
  d.kw = 1;

  size_t blob_size = 0, smem = 0;
  size_t rec = 16, tsp = 0, tbd = 0;
  std::vector<std::vector<uint32_t>> streams(job.n_sublattices);
  std::vector<std::pair<std::vector<uint32_t>, std::vector<uint32_t>>> k2_data;
  std::vector<std::vector<uint32_t>> k2_nbp_data;
  for (uint32_t p = 0; p < job.n_sublattices; ++p) {
    const sqsg_sublattice& sl = job.sublattices[p];
    PartDesc& P = d.parts[p];
    if (sl.n_sites == 0) throw std::invalid_argument("empty structure");
    if (sl.n_species == 0 || sl.n_shells == 0) throw std::out_of_range("no coordination shells selected");
    if (sl.n_species > static_cast<uint32_t>(kMaxSpecies))
      throw unsupported_error("more than 8 species in one optimised structure");
    if (sl.n_shells > 255) throw unsupported_error("more than 255 shells");
    if (!sl.species || !sl.prefactors || !sl.pair_weights || !sl.target || (sl.n_pairs && !sl.pairs))
      throw std::invalid_argument("null array in sublattice");
    if (sl.n_windows == 0 || !sl.windows) throw std::invalid_argument("no shuffle window");
    if (sl.n_windows > static_cast<uint32_t>(kMaxWindows)) throw unsupported_error("more than 16 shuffle windows");
    for (uint32_t x = 0; x < sl.n_sites; ++x)
      if (sl.species[x] >= sl.n_species) throw std::out_of_range("packed species index >= n_species");
    for (uint32_t w = 0; w < sl.n_windows; ++w) {
      if (sl.windows[2 * w] >= sl.windows[2 * w + 1] || sl.windows[2 * w + 1] > sl.n_sites)
        throw std::out_of_range("invalid shuffle window");
      if (w > 0 && sl.windows[2 * w] < sl.windows[2 * w - 1]) throw std::invalid_argument("overlapping windows");
    }
    if (pj.systematic && sl.n_windows != 1)
      throw std::invalid_argument("In \"systematic\" iteration mode only one sublattice is allowed");
    P.n_sites = sl.n_sites;
    P.n_species = sl.n_species;
    P.n_shells = sl.n_shells;
    P.n_windows = sl.n_windows;
    P.hw = (sl.n_species + 1) / 2;
    if (sl.n_species > 4) d.kw = 2;
    streams[p] = build_stream(sl);
    P.stream_words = static_cast<uint32_t>(streams[p].size());
    P.stream_narrow = narrow_stream(sl.n_sites) ? 1u : 0u;
    const size_t skk = static_cast<size_t>(sl.n_shells) * sl.n_species * sl.n_species;
    // binary fast path data: per (shell, site) mask of the neighbours j > i (bit N-1-j)
    const bool k2 = job.n_sublattices == 1 && sl.n_species == 2 && sl.n_sites <= 64 && sl.n_shells <= kK2MaxShells &&
                    job.keep < 32 && option(kOptForceGeneral) == 0;
    std::vector<uint32_t> k2_entries, k2_shells, k2_nbp;
    if (k2) {
      const uint32_t N = sl.n_sites;
      std::vector<unsigned long long> nb(static_cast<size_t>(sl.n_shells) * N, 0ull);
      std::vector<uint32_t> ps(sl.n_shells, 0);
      for (uint32_t e = 0; e < sl.n_pairs; ++e) {
        uint32_t i = sl.pairs[3 * e], j = sl.pairs[3 * e + 1];
        const uint32_t sh = sl.pairs[3 * e + 2];
        if (i > j) std::swap(i, j);
        nb[static_cast<size_t>(sh) * N + i] |= 1ull << (N - 1 - j);
        ps[sh]++;
      }
      std::vector<uint32_t> shell_end(sl.n_shells);
      for (uint32_t sh = 0; sh < sl.n_shells; ++sh) {
        for (uint32_t i = 0; i < N; ++i) {
          const unsigned long long m = nb[static_cast<size_t>(sh) * N + i];
          if (!m) continue;
          k2_entries.push_back(static_cast<uint32_t>(m));
          k2_entries.push_back(static_cast<uint32_t>(m >> 32));
          k2_entries.push_back(N - 1 - i);
          k2_entries.push_back(static_cast<uint32_t>(__builtin_popcountll(m)));
        }
        shell_end[sh] = static_cast<uint32_t>(k2_entries.size() / 4);
      }
      uint32_t ones = 0;
      for (uint32_t x = 0; x < N; ++x) ones += sl.species[x] != 0 ? 1u : 0u;
      // degree classes: sites grouped by their number of shell-s pairs (either end), so that
      // n01 + n10 = sum_x b_x deg_s(x) - 2 n11 costs one popcount per class. The number of ones is
      // the same in every configuration, so the largest class c* needs none: the sum is
      // deg_c* * ones + sum over the other classes of (deg_c - deg_c*) * popc (mod 2^32), and a
      // lattice whose sites all have one degree (every Bravais lattice) needs no popcount at all.
      for (uint32_t sh = 0; sh < sl.n_shells; ++sh) {
        std::vector<uint32_t> deg(N, 0);
        for (uint32_t i = 0; i < N; ++i) {
          const unsigned long long m = nb[static_cast<size_t>(sh) * N + i];
          deg[i] += static_cast<uint32_t>(__builtin_popcountll(m));
          for (uint32_t j = 0; j < N; ++j)
            if ((m >> (N - 1 - j)) & 1ull) deg[j]++;
        }
        std::map<uint32_t, unsigned long long> classes;  // degree 0 included: the classes cover all sites
        for (uint32_t x = 0; x < N; ++x) classes[deg[x]] |= 1ull << (N - 1 - x);
        uint32_t dstar = 0;
        int best = -1;
        for (auto& [dv, m] : classes)
          if (__builtin_popcountll(m) > best) best = __builtin_popcountll(m), dstar = dv;
        const uint32_t d0 = static_cast<uint32_t>(k2_entries.size() / 4);
        for (auto& [dv, m] : classes) {
          if (dv == dstar) continue;
          k2_entries.push_back(static_cast<uint32_t>(m));
          k2_entries.push_back(static_cast<uint32_t>(m >> 32));
          k2_entries.push_back(dv - dstar);
          k2_entries.push_back(0);
        }
        k2_shells.push_back(ps[sh]);
        k2_shells.push_back(shell_end[sh]);
        k2_shells.push_back(d0);
        k2_shells.push_back(static_cast<uint32_t>(k2_entries.size() / 4));
        k2_shells.push_back(dstar * ones);
        for (int pad = 0; pad < 3; ++pad) k2_shells.push_back(0);
      }
      // neighbour masks indexed by the bit position p = N-1-i of site i, for the per-configuration
      // loop over the set bits of the minority species
      const uint32_t slots = N <= 32 ? 32 : 64;
      for (uint32_t sh = 0; sh < sl.n_shells; ++sh)
        for (uint32_t bp = 0; bp < slots; ++bp) {
          const unsigned long long m = bp < N ? nb[static_cast<size_t>(sh) * N + (N - 1 - bp)] : 0ull;
          k2_nbp.push_back(static_cast<uint32_t>(m));
          if (slots == 64) k2_nbp.push_back(static_cast<uint32_t>(m >> 32));
        }
      P.k2_zeros = 2 * ones > N ? 1u : 0u;
    }
    // blob section layout: cubes | windows | species codes | binary-path masks | pair stream. The
    // stream is staged into shared memory with the rest when that costs no CTA per SM; otherwise
    // (large cells, split jobs, the binary path that does not read it) it is read from the blob
    // through L1: one copy per SM for all its CTAs, leaving the shared memory to more CTAs.
    size_t off = 0;
    P.cube_off = 0;
    off = align_up(3 * skk * pj.tsz, 16);
    P.win_off = static_cast<uint32_t>(off);
    off = align_up(off + 8ull * sl.n_windows, 16);
    P.species_off = static_cast<uint32_t>(off);
    off = align_up(off + sl.n_sites, 16);
    if (k2) {
      P.k2_off = static_cast<uint32_t>(off);
      P.k2_entries = static_cast<uint32_t>(k2_entries.size() / 4);
      off = align_up(off + 4 * k2_entries.size(), 16);
      P.k2_shell_off = static_cast<uint32_t>(off);
      off = align_up(off + 4 * k2_shells.size(), 16);
      P.k2_nbp_off = static_cast<uint32_t>(off);
      off = align_up(off + 4 * k2_nbp.size(), 16);
      k2_data.emplace_back(std::move(k2_entries), std::move(k2_shells));
      k2_nbp_data.emplace_back(std::move(k2_nbp));
    } else {
      k2_data.emplace_back();
      k2_nbp_data.emplace_back();
    }
    P.stream_off = static_cast<uint32_t>(off);
    const size_t with_stream = align_up(off + 4ull * streams[p].size(), 16);
    const size_t lanes = (static_cast<size_t>((sl.n_sites + 3) / 4) +
                          static_cast<size_t>(sl.n_shells) * sl.n_species * P.hw) * kBlock * 4;
    const bool staged = !k2 && job.n_sublattices == 1 &&
                        ctas_per_sm(job.device, with_stream + lanes) >= ctas_per_sm(job.device, off + lanes);
    P.stream_global = staged ? 0u : 1u;
    P.static_bytes = static_cast<uint32_t>(staged ? with_stream : off);
    P.blob_off = static_cast<uint32_t>(blob_size);
    blob_size += with_stream;
    off = P.static_bytes;
    // shared memory: staged section, species columns, histogram
    P.smem_off = static_cast<uint32_t>(smem);
    P.col_off = static_cast<uint32_t>(off);
    off += static_cast<size_t>((sl.n_sites + 3) / 4) * kBlock * 4;
    P.hist_off = static_cast<uint32_t>(off);
    off += static_cast<size_t>(sl.n_shells) * sl.n_species * P.hw * kBlock * 4;
    smem += align_up(off, 16);
    // candidate record layout
    P.rec_species_off = static_cast<uint32_t>(rec);
    rec = align_up(rec + sl.n_sites, 8);
    P.rec_obj_off = static_cast<uint32_t>(rec);
    rec += 8;
    P.rec_sro_off = static_cast<uint32_t>(rec);
    rec = align_up(rec + skk * pj.tsz, 8);
    P.trace_species_off = static_cast<uint32_t>(tsp);
    tsp += sl.n_sites;
    P.trace_bonds_off = static_cast<uint32_t>(tbd);
    tbd += skk;
    pj.parts.push_back(PartMeta{sl.n_sites, sl.n_species, sl.n_shells});
    if (pj.systematic) pj.total = window_permutations(sl, P);
    if (k2 && (!pj.systematic || (P.unrank_k == 2 && P.unrank_rev[0] == 0 && P.unrank_rev[1] == 1)))
      d.k2 = sl.n_sites <= 32 ? 1 : 2;
  }
  if (!pj.systematic) pj.total = job.iterations;
  d.total = pj.total;
  if (job.range_first > pj.total) throw std::out_of_range("range_first beyond the configuration space");
  pj.range_first = job.range_first;
  pj.range_count = job.range_count ? job.range_count : pj.total - job.range_first;
  if (pj.range_count > pj.total - pj.range_first) throw std::out_of_range("range beyond the configuration space");
  d.trace_base = pj.range_first + (pj.systematic ? 1 : 0);
  d.record_bytes = static_cast<uint32_t>(align_up(rec, 16));
  pj.record_bytes = d.record_bytes;
  d.smem_full = static_cast<uint32_t>(smem);
  // keep >= 32: each warp's best list (keep+1 entries, rounded up to whole rows of 32) lives in shared
  // memory after the parts; smaller keep uses one register per lane
  if (job.keep >= 32) {
    d.big_len = static_cast<uint32_t>(align_up(job.keep + 1, 32));
    d.big_off = static_cast<uint32_t>(align_up(smem, 16));
    smem = d.big_off + static_cast<size_t>(kBlock / 32) * d.big_len * sizeof(double);
  }
  d.smem_bytes = static_cast<uint32_t>(smem);
  d.trace = trace_capacity > 0 ? 1 : 0;
  d.trace_capacity = trace_capacity;
  d.trace_species_stride = static_cast<uint32_t>(tsp);
  d.trace_bonds_stride = static_cast<uint32_t>(tbd);
  d.wait_ns = static_cast<uint64_t>(std::max<long long>(1000, option(kOptStageWaitNs)));
  d.debug = option(kOptDebugSkipStaging) ? kDebugSkipStaging : 0u;
  if (job.has_seed) {
    d.seed = job.seed;
  } else {
    std::random_device rd;  // core/shuffle.h:16-21 draws an unseeded run's seed the same way
    d.seed = (static_cast<uint64_t>(rd()) << 32) ^ rd();
  }
  pj.blob.assign(blob_size, 0);
  for (uint32_t p = 0; p < job.n_sublattices; ++p) {
    const sqsg_sublattice& sl = job.sublattices[p];
    const PartDesc& P = d.parts[p];
    const size_t skk = static_cast<size_t>(sl.n_shells) * sl.n_species * sl.n_species;
    uint8_t* base = pj.blob.data() + P.blob_off;
    std::memcpy(base + P.cube_off, sl.prefactors, skk * pj.tsz);
    std::memcpy(base + P.cube_off + skk * pj.tsz, sl.pair_weights, skk * pj.tsz);
    std::memcpy(base + P.cube_off + 2 * skk * pj.tsz, sl.target, skk * pj.tsz);
    std::memcpy(base + P.win_off, sl.windows, 8ull * sl.n_windows);
    std::memcpy(base + P.stream_off, streams[p].data(), 4ull * streams[p].size());
    for (uint32_t x = 0; x < sl.n_sites; ++x) base[P.species_off + x] = static_cast<uint8_t>(sl.species[x] << 3);
    const auto& k2d = k2_data[p];
    if (!k2d.first.empty()) std::memcpy(base + P.k2_off, k2d.first.data(), 4 * k2d.first.size());
    if (!k2d.second.empty()) std::memcpy(base + P.k2_shell_off, k2d.second.data(), 4 * k2d.second.size());
    if (!k2_nbp_data[p].empty())
      std::memcpy(base + P.k2_nbp_off, k2_nbp_data[p].data(), 4 * k2_nbp_data[p].size());
  }
  // binary systematic path: binomials C(m, j) for m <= window size, j <= ones in the window, kept in
  // global memory after the staged sections (read through the L1 by the per-thread unrank)
  if (d.k2 && pj.systematic) {
    PartDesc& P = d.parts[0];
    const uint32_t n = job.sublattices[0].windows[1] - job.sublattices[0].windows[0];
    const uint32_t ones = P.unrank_hist[1], cols = ones + 1;
    const size_t off = align_up(pj.blob.size(), 16);
    pj.blob.resize(off + 8ull * (n + 1) * cols, 0);
    P.k2_binom_off = static_cast<uint32_t>(off);
    unsigned long long* b = reinterpret_cast<unsigned long long*>(pj.blob.data() + off);
    for (uint32_t m = 0; m <= n; ++m)
      for (uint32_t j = 0; j <= ones; ++j)
        b[m * cols + j] = (j == 0) ? 1ull : (m == 0 ? 0ull : b[(m - 1) * cols + j - 1] + b[(m - 1) * cols + j]);
  }
  return pj;
}


void make_tiles(PreparedJob& pj, uint32_t job_index, std::vector<Tile>& tiles, uint64_t max_per_thread) {
  size_t added = 0;
  for_each_tile(
      pj.range_first, pj.range_count, pj.systematic,
      [&](Tile t) -> bool {
        if (++added > kMaxJobTiles) return false;
        t.job = job_index;
        tiles.push_back(t);
        return true;
      },
      max_per_thread);
  if (added > kMaxJobTiles)
    throw unsupported_error("the job has more than " + std::to_string(kMaxJobTiles) +
                            " tiles; split it with range_first/range_count");
}

}  // namespace sqsg
