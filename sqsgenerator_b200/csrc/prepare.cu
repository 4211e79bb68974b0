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
#include <array>
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

// Draw word of a random-mode window with exactly two species: m (the rarer species' sites, ties to the
// higher species index) | its code << 16 | the other code << 24; 0 for any other window, which takes
// the Fisher-Yates shuffle.
static uint32_t floyd_word(const sqsg_sublattice& sl, uint32_t w) {
  const uint32_t lo = sl.windows[2 * w], hi = sl.windows[2 * w + 1];
  uint32_t counts[kMaxSpecies] = {0};
  for (uint32_t x = lo; x < hi; ++x) counts[sl.species[x]]++;
  uint32_t present[kMaxSpecies], distinct = 0;  // species of the window, ascending
  for (uint32_t v = 0; v < static_cast<uint32_t>(kMaxSpecies); ++v)
    if (counts[v]) present[distinct++] = v;
  if (distinct != 2) return 0u;
  const uint32_t a = present[0], b = present[1];
  const uint32_t rare = counts[b] <= counts[a] ? b : a, other = rare == a ? b : a;
  if (counts[rare] > 0xffffu) return 0u;
  return counts[rare] | (rare << 3) << 16 | (other << 3) << 24;
}

// Lattice-path tables of one part, from its supercell hint (sqsg_sublattice::lattice): valid only
// when the sites are a bijection onto (unit-cell site, cell) and every pair belongs to a translation
// class {(beta, c), (beta2, c + d)} that the pair list holds completely — once per cell, or once per
// pair of cells for a class that is its own reverse (beta == beta2, 2d = 0).
struct LatticeTables {
  uint32_t m = 0, A = 0, B = 0, C = 0, cells = 0, chunks = 0, words = 1;
  unsigned long long full[2] = {0, 0};
  std::vector<uint32_t> site_off;  // m x 4*chunks column offsets (cells past the grid repeat cell 0)
  std::vector<uint32_t> ent;       // beta | beta2 << 4 | translation << 8
  std::vector<uint32_t> shell;     // per shell: first class, first self-reverse class, end, pairs
  std::vector<LatTr> tr;
  std::vector<uint32_t> deg;       // S x m
};

static bool lattice_tables(const sqsg_sublattice& sl, LatticeTables& L) {
  if (!sl.lattice) return false;
  const uint32_t N = sl.n_sites, S = sl.n_shells;
  const uint32_t A = sl.cells[0], B = sl.cells[1], C = sl.cells[2], m = sl.n_basis;
  if (A == 0 || B == 0 || C == 0 || m == 0 || m > 15) return false;
  const uint64_t cells = static_cast<uint64_t>(A) * B * C;
  if (cells > 128 || cells * m != N) return false;
  std::vector<uint32_t> beta(N), cx(N), cy(N), cz(N), site_at(N, ~0u);
  for (uint32_t x = 0; x < N; ++x) {
    const uint32_t* h = sl.lattice + 4 * static_cast<size_t>(x);
    if (h[0] >= m || h[1] >= A || h[2] >= B || h[3] >= C) return false;
    beta[x] = h[0];
    cx[x] = h[1];
    cy[x] = h[2];
    cz[x] = h[3];
    const uint32_t q = h[0] * static_cast<uint32_t>(cells) + h[1] + A * (h[2] + B * h[3]);
    if (site_at[q] != ~0u) return false;
    site_at[q] = x;
  }
  // class key: shell, beta, beta2, displacement (dx + 64 * (dy + 64 * dz)) of the second site
  auto key_of = [](uint32_t s, uint32_t b1, uint32_t b2, uint32_t dx, uint32_t dy, uint32_t dz) {
    return (static_cast<unsigned long long>((s << 8) | (b1 << 4) | b2) << 18) | (dx + 64u * (dy + 64u * dz));
  };
  std::vector<std::pair<unsigned long long, uint32_t>> member(sl.n_pairs);  // (class key, cell id in class)
  std::vector<uint8_t> self_rev(sl.n_pairs);
  for (uint32_t e = 0; e < sl.n_pairs; ++e) {
    const uint32_t i = sl.pairs[3 * e], j = sl.pairs[3 * e + 1], s = sl.pairs[3 * e + 2];
    const uint32_t dx = (cx[j] + A - cx[i]) % A, dy = (cy[j] + B - cy[i]) % B, dz = (cz[j] + C - cz[i]) % C;
    const unsigned long long k1 = key_of(s, beta[i], beta[j], dx, dy, dz);
    const unsigned long long k2 = key_of(s, beta[j], beta[i], (A - dx) % A, (B - dy) % B, (C - dz) % C);
    const uint32_t ci = cx[i] + A * (cy[i] + B * cz[i]), cj = cx[j] + A * (cy[j] + B * cz[j]);
    if (k1 == k2) {
      member[e] = {k1, std::min(ci, cj)};
      self_rev[e] = 1;
    } else {
      member[e] = k1 < k2 ? std::make_pair(k1, ci) : std::make_pair(k2, cj);
    }
  }
  std::vector<uint32_t> order(sl.n_pairs);
  for (uint32_t e = 0; e < sl.n_pairs; ++e) order[e] = e;
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return member[a] < member[b]; });
  struct Class {
    unsigned long long key;
    bool self;
    uint32_t count;
  };
  std::vector<Class> classes;
  for (size_t k = 0; k < order.size(); ++k) {
    const auto& mk = member[order[k]];
    if (k > 0 && member[order[k - 1]] == mk) return false;  // the same pair twice
    if (classes.empty() || classes.back().key != mk.first)
      classes.push_back(Class{mk.first, self_rev[order[k]] != 0, 0});
    classes.back().count++;
  }
  for (auto& c : classes)
    if (c.count != (c.self ? cells / 2 : cells)) return false;  // an incomplete class
  L.m = m;
  L.A = A;
  L.B = B;
  L.C = C;
  L.cells = static_cast<uint32_t>(cells);
  L.chunks = (L.cells + 3) / 4;
  L.words = cells > 64 ? 2 : 1;
  for (uint32_t c = 0; c < L.cells; ++c) L.full[c / 64] |= 1ull << (c % 64);
  L.site_off.assign(static_cast<size_t>(m) * 4 * L.chunks, 0);
  for (uint32_t b = 0; b < m; ++b)
    for (uint32_t c = 0; c < 4 * L.chunks; ++c)
      L.site_off[b * 4 * L.chunks + c] = host_site_off(site_at[b * L.cells + (c < L.cells ? c : 0)]);
  // translations: the second site's planes move by -d onto the first site's cells
  std::map<uint32_t, uint32_t> tr_index;
  auto translation = [&](uint32_t dpack) -> uint32_t {
    const uint32_t dx = dpack % 64, dy = (dpack / 64) % 64, dz = dpack / 4096;
    const uint32_t tx = (A - dx) % A, ty = (B - dy) % B, tz = (C - dz) % C;
    const uint32_t tkey = tx + 64u * (ty + 64u * tz);
    auto it = tr_index.find(tkey);
    if (it != tr_index.end()) return it->second;
    LatTr t{};
    t.sx = tx;
    t.sxr = A - tx;
    t.sy = A * ty;
    t.syr = A * B - A * ty;
    t.sz = A * B * tz;
    t.szr = L.cells - A * B * tz;
    for (uint32_t c = 0; c < L.cells; ++c) {
      const uint32_t x = c % A, y = (c / A) % B;
      const unsigned long long bit = 1ull << (c % 64);
      if (x >= tx) t.mxh[c / 64] |= bit;
      if (y >= ty) t.myh[c / 64] |= bit;
    }
    const uint32_t idx = static_cast<uint32_t>(L.tr.size());
    L.tr.push_back(t);
    tr_index[tkey] = idx;
    return idx;
  };
  L.shell.assign(4 * static_cast<size_t>(S), 0);
  L.deg.assign(static_cast<size_t>(S) * m, 0);
  for (uint32_t s = 0; s < S; ++s) {
    std::vector<std::pair<uint64_t, uint32_t>> normal, self;  // (sort key, entry)
    uint32_t pairs = 0;
    // A class {(beta, c), (beta2, c + d)} counts the same pairs when read from either end: as beta's
    // planes against beta2's translated by -d, or beta2's against beta's translated by +d. Each
    // distinct (translated site, translation) costs one translation of its planes per configuration,
    // so the ends are chosen greedily to share as few of them as possible.
    struct Option {
      uint32_t beta, beta2, dpack;
      uint64_t key;  // translated site and translation
    };
    auto option_of = [&](uint32_t b1, uint32_t b2, uint32_t dpack) {
      const uint32_t dx = dpack % 64, dy = (dpack / 64) % 64, dz = dpack / 4096;
      const uint64_t tkey = (A - dx) % A + 64ull * ((B - dy) % B + 64ull * ((C - dz) % C));
      return Option{b1, b2, dpack, b2 | (tkey << 4)};
    };
    auto negate = [&](uint32_t dpack) {
      const uint32_t dx = dpack % 64, dy = (dpack / 64) % 64, dz = dpack / 4096;
      return (A - dx) % A + 64u * ((B - dy) % B + 64u * ((C - dz) % C));
    };
    std::vector<std::array<Option, 2>> opts;
    for (auto& c : classes) {
      const uint32_t cs = static_cast<uint32_t>(c.key >> 26);
      if (cs != s) continue;
      const uint32_t b1 = static_cast<uint32_t>(c.key >> 22) & 0xfu, b2 = static_cast<uint32_t>(c.key >> 18) & 0xfu;
      const uint32_t dpack = static_cast<uint32_t>(c.key & 0x3ffffull);
      pairs += c.count;
      L.deg[s * m + b1] += 1;
      if (!c.self) L.deg[s * m + b2] += 1;
      if (c.self) {  // its own reverse: either end gives the same entry
        const uint32_t en = b1 | (b2 << 4) | (translation(dpack) << 8);
        self.emplace_back((static_cast<uint64_t>(en >> 4) << 4) | b1, en);
      } else {
        opts.push_back({option_of(b1, b2, dpack), option_of(b2, b1, negate(dpack))});
      }
    }
    std::vector<int> pick(opts.size(), -1);
    for (size_t left = opts.size(); left > 0;) {
      std::map<uint64_t, uint32_t> freq;
      for (size_t k = 0; k < opts.size(); ++k)
        if (pick[k] < 0) {
          freq[opts[k][0].key]++;
          if (opts[k][1].key != opts[k][0].key) freq[opts[k][1].key]++;
        }
      uint64_t best = 0;
      uint32_t best_n = 0;
      for (auto& [key, cnt] : freq)  // most shared first; ties: the smaller key (deterministic)
        if (cnt > best_n) best = key, best_n = cnt;
      for (size_t k = 0; k < opts.size(); ++k)
        if (pick[k] < 0 && (opts[k][0].key == best || opts[k][1].key == best)) {
          pick[k] = opts[k][0].key == best ? 0 : 1;
          --left;
        }
    }
    for (size_t k = 0; k < opts.size(); ++k) {
      const Option& o = opts[k][pick[k]];
      const uint32_t en = o.beta | (o.beta2 << 4) | (translation(o.dpack) << 8);
      // classes sharing (beta2, translation) are adjacent: their translated planes are computed once
      normal.emplace_back((static_cast<uint64_t>(en >> 4) << 4) | o.beta, en);
    }
    std::sort(normal.begin(), normal.end());
    std::sort(self.begin(), self.end());
    L.shell[4 * s] = static_cast<uint32_t>(L.ent.size());
    for (auto& x : normal) L.ent.push_back(x.second);
    L.shell[4 * s + 1] = static_cast<uint32_t>(L.ent.size());
    for (auto& x : self) L.ent.push_back(x.second);
    L.shell[4 * s + 2] = static_cast<uint32_t>(L.ent.size());
    L.shell[4 * s + 3] = pairs;
  }
  return L.tr.size() < (1u << 24);
}

// ------------------------------------------------------------------------------------------------
// Tuning table
struct TableEntry {
  uint64_t key;
  int path, stage;
  uint32_t ctas, tile_cap;
};
static const TableEntry kShippedTable[] = {
#include "tuning_table.inc"
    {0, -1, -1, 0, 0}};

static std::mutex g_tuning_mutex;
static std::map<uint64_t, Tuning>& tuning_cache() {
  static auto* m = new std::map<uint64_t, Tuning>();  // never destroyed: used until exit
  return *m;
}

static uint32_t ceil_log2(uint64_t v) {
  uint32_t b = 0;
  while ((1ull << b) < v && b < 63) ++b;
  return b;
}

uint64_t bucket_key(const sqsg_job& job) {
  uint64_t n = 0, p = 0;
  uint32_t kmax = 0, smax = 0, hint = 0;
  for (uint32_t k = 0; k < job.n_sublattices && job.sublattices; ++k) {
    const sqsg_sublattice& sl = job.sublattices[k];
    n += sl.n_sites;
    p += sl.n_pairs;
    kmax = std::max(kmax, sl.n_species);
    smax = std::max(smax, sl.n_shells);
    hint |= sl.lattice ? 1u : 0u;
  }
  uint64_t key = static_cast<uint64_t>(job.prec & 1);
  key = (key << 1) | static_cast<uint64_t>(job.iteration_mode & 1);
  key = (key << 4) | std::min<uint32_t>(job.n_sublattices, 15);
  key = (key << 4) | std::min<uint32_t>(kmax, 15);
  key = (key << 8) | std::min<uint32_t>(smax, 255);
  key = (key << 6) | ceil_log2(n);
  key = (key << 6) | ceil_log2(p);
  key = (key << 1) | hint;
  return key + 1;  // 0 ends the shipped table
}

bool tuning_lookup(uint64_t key, Tuning& out) {
  {
    std::lock_guard<std::mutex> l(g_tuning_mutex);
    auto it = tuning_cache().find(key);
    if (it != tuning_cache().end()) {
      out = it->second;
      return true;
    }
  }
  for (const TableEntry& e : kShippedTable)
    if (e.key == key) {
      out = Tuning{e.path, e.stage, e.ctas, e.tile_cap};
      return true;
    }
  return false;
}

void tuning_store(uint64_t key, const Tuning& t) {
  std::lock_guard<std::mutex> l(g_tuning_mutex);
  tuning_cache()[key] = t;
}

PreparedJob prepare(const sqsg_job& job, uint64_t trace_capacity, const Tuning* tuning) {
  PreparedJob pj;
  if (tuning)
    pj.tuning = *tuning;
  else if (option(kOptUseTuning))
    tuning_lookup(bucket_key(job), pj.tuning);
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

  size_t blob_size = 0, smem = 0, engine_end = 0;
  size_t rec = 16, tsp = 0, tbd = 0;
  std::vector<std::vector<uint32_t>> streams(job.n_sublattices);
  std::vector<std::pair<std::vector<uint32_t>, std::vector<uint32_t>>> k2_data;
  std::vector<std::vector<uint32_t>> k2_nbp_data;
  // validation, pair streams and lattice tables of every part first: the path is chosen per job
  std::vector<LatticeTables> lat(job.n_sublattices);
  // reference-stream debug mode: random jobs only, on the pair-stream path
  pj.chain = !pj.systematic && option(kOptRapidrand) != 0;
  bool job_lat = option(kOptForceGeneral) == 0 && !pj.chain;
  bool will_k2 = false;
  for (uint32_t p = 0; p < job.n_sublattices; ++p) {
    const sqsg_sublattice& sl = job.sublattices[p];
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
    streams[p] = build_stream(sl);  // validates the pair list
    job_lat = job_lat && lattice_tables(sl, lat[p]) && sl.n_species >= 2;
    // two-word cell sets (65..128 cells) run in sqsg_engine_latw, which holds up to five species;
    // every part of a job uses the same width
    job_lat = job_lat && (lat[p].words == 1 || sl.n_species <= 5) && lat[p].words == lat[0].words;
    if (job.n_sublattices == 1 && sl.n_species == 2 && sl.n_sites <= 64 && sl.n_shells <= kK2MaxShells &&
        job.keep < 32 && option(kOptForceGeneral) == 0 && !pj.chain) {
      bool has0 = false, has1 = false;  // systematic: the window must hold both species
      for (uint32_t x = sl.windows[0]; x < sl.windows[1]; ++x) (sl.species[x] ? has1 : has0) = true;
      will_k2 = !pj.systematic || (has0 && has1);
    }
  }
  job_lat = job_lat && !will_k2 && pj.tuning.path != SQSG_PATH_GENERAL;
  d.lat = job_lat ? 1u : 0u;
  for (uint32_t p = 0; p < job.n_sublattices; ++p) {
    const sqsg_sublattice& sl = job.sublattices[p];
    PartDesc& P = d.parts[p];
    P.n_sites = sl.n_sites;
    P.n_species = sl.n_species;
    P.n_shells = sl.n_shells;
    P.n_windows = sl.n_windows;
    for (uint32_t x = 0; x < sl.n_sites; ++x) P.ones += sl.species[x] == 1 ? 1u : 0u;
    P.hw = (sl.n_species + 1) / 2;
    if (sl.n_species > 4) d.kw = 2;
    P.stream_words = static_cast<uint32_t>(streams[p].size());
    P.stream_narrow = narrow_stream(sl.n_sites) ? 1u : 0u;
    const size_t skk = static_cast<size_t>(sl.n_shells) * sl.n_species * sl.n_species;
    // binary fast path data: per (shell, site) mask of the neighbours j > i (bit N-1-j)
    const bool k2 = will_k2;
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
    off = align_up(off + 12ull * sl.n_windows, 16);
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
    const LatticeTables& LT = lat[p];
    size_t planes = 0;  // lattice path: per-lane plane bytes
    if (job_lat) {
      P.lat_km = sl.n_species <= 5 ? sl.n_species : 8u;
      d.lat_kmax = std::max(d.lat_kmax, P.lat_km);
      P.lat_basis = LT.m;
      P.lat_cells = LT.cells;
      P.lat_chunks = LT.chunks;
      P.lat_full = LT.full[0];
      P.lat_full_hi = LT.full[1];
      d.lat_words = LT.words;
      P.lat_site_off = static_cast<uint32_t>(off);
      off = align_up(off + 4 * LT.site_off.size(), 16);
      P.lat_ent_off = static_cast<uint32_t>(off);
      off = align_up(off + 4 * LT.ent.size(), 16);
      P.lat_shell_off = static_cast<uint32_t>(off);
      off = align_up(off + 4 * LT.shell.size(), 16);
      P.lat_tr_off = static_cast<uint32_t>(off);
      off = align_up(off + (LT.words == 1 ? sizeof(LatTrW<1>) : sizeof(LatTrW<2>)) * LT.tr.size(), 16);
      P.lat_deg_off = static_cast<uint32_t>(off);
      off = align_up(off + 4 * LT.deg.size(), 16);
      planes = static_cast<size_t>(LT.m) * (sl.n_species - 1) * 8 * LT.words * kBlock;
    }
    P.stream_off = static_cast<uint32_t>(off);
    const size_t with_stream = align_up(off + 4ull * streams[p].size(), 16);
    const size_t lanes = (static_cast<size_t>((sl.n_sites + 3) / 4) +
                          static_cast<size_t>(sl.n_shells) * sl.n_species * P.hw) * kBlock * 4;
    // the lattice path reads the stream only for traces and rebuilt records: never staged
    bool staged = !k2 && !job_lat && job.n_sublattices == 1 &&
                  ctas_per_sm(job.device, with_stream + lanes) >= ctas_per_sm(job.device, off + lanes);
    if (!k2 && !job_lat && job.n_sublattices == 1 && pj.tuning.stage >= 0)  // a measured choice
      staged = pj.tuning.stage == 1 && ctas_per_sm(job.device, with_stream + lanes) >= 1;
    P.stream_global = staged ? 0u : 1u;
    P.static_bytes = static_cast<uint32_t>(staged ? with_stream : off);
    P.blob_off = static_cast<uint32_t>(blob_size);
    blob_size += with_stream;
    off = P.static_bytes;
    // shared memory: staged section, species columns, histogram
    P.smem_off = static_cast<uint32_t>(smem);
    P.col_off = static_cast<uint32_t>(off);
    off += static_cast<size_t>((sl.n_sites + 3) / 4) * kBlock * 4;
    if (job_lat) {
      off = align_up(off, 16);
      P.lat_planes_off = static_cast<uint32_t>(off);
      off += planes;
    }
    P.hist_off = static_cast<uint32_t>(off);
    engine_end = smem + off;  // the lattice path needs no histogram (but traces and rebuilt records do)
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
    pj.parts.push_back(PartMeta{sl.n_sites, sl.n_species, sl.n_shells, sl.n_pairs});
    if (pj.systematic) pj.total = window_permutations(sl, P);
    if (k2 && (!pj.systematic || (P.unrank_k == 2 && P.unrank_rev[0] == 0 && P.unrank_rev[1] == 1)))
      d.k2 = sl.n_sites <= 32 ? 1 : 2;
  }
  if (!pj.systematic) pj.total = job.iterations;
  if (pj.chain) {
    // The reference's thread-pool blocks over [0, iterations) (BS_thread_pool v5 blocks, sqs.h:461-466):
    // iterations / chunk_size blocks (at least one), the remainder spread one by one over the first.
    if (job.range_first != 0 || (job.range_count != 0 && job.range_count != job.iterations))
      throw unsupported_error("the rapidrand debug mode runs whole jobs (no range_first/range_count)");
    const uint64_t total = job.iterations;
    uint64_t nb = job.chunk_size ? total / job.chunk_size : 0;
    if (nb == 0) nb = 1;
    nb = std::max<uint64_t>(1, std::min<uint64_t>(nb, std::max<uint64_t>(total, 1)));
    d.chain = 1;
    d.chain_split = job.sublattice_mode == 1 ? 1u : 0u;
    d.chain_blocks = nb;
    d.chain_block = total / nb;
    d.chain_rem = total % nb;
    for (uint32_t p = 0; p < job.n_sublattices; ++p) {
      const sqsg_sublattice& sl = job.sublattices[p];
      uint32_t draws = 0;
      for (uint32_t w = 0; w < sl.n_windows; ++w) draws += sl.windows[2 * w + 1] - sl.windows[2 * w] - 1;
      d.parts[p].chain_draws = draws;
    }
  }
  // Random mode: exact configuration keys for a deduplicating re-run (see column_key), when the
  // product of the parts' arrangement counts stays within kDedupMaxSpace.
  if (!pj.systematic && trace_capacity == 0) {
    unsigned __int128 prod = 1;
    bool ok = true;
    for (uint32_t p = 0; p < job.n_sublattices && ok; ++p) {
      const sqsg_sublattice& sl = job.sublattices[p];
      PartDesc& P = d.parts[p];
      uint32_t counts[kMaxSpecies] = {};
      for (uint32_t x = 0; x < sl.n_sites; ++x) counts[sl.species[x]]++;
      unsigned __int128 m = 1;  // multinomial(n; counts) as a product of binomials, exact at every step
      uint64_t seen = 0;
      for (uint32_t k = 0; k < sl.n_species && ok; ++k)
        for (uint32_t i = 1; i <= counts[k] && ok; ++i) {
          m = m * (++seen) / i;
          ok = m <= kDedupMaxSpace;
        }
      if (!ok) break;
      for (uint32_t k = 0; k < kMaxSpecies; ++k) P.dd_counts[k] = counts[k];
      P.dd_space = static_cast<unsigned long long>(m);
      P.dd_stride = static_cast<unsigned long long>(prod);
      prod *= m;
      ok = prod <= kDedupMaxSpace;
    }
    pj.dedup_ok = ok;
    pj.dedup_space = ok ? static_cast<uint64_t>(prod) : 0;
  }
  d.total = pj.total;
  if (job.range_first > pj.total) throw std::out_of_range("range_first beyond the configuration space");
  pj.range_first = job.range_first;
  pj.range_count = job.range_count ? job.range_count : pj.total - job.range_first;
  if (pj.range_count > pj.total - pj.range_first) throw std::out_of_range("range beyond the configuration space");
  d.trace_base = pj.range_first + (pj.systematic ? 1 : 0);
  d.record_bytes = static_cast<uint32_t>(align_up(rec, 16));
  pj.record_bytes = d.record_bytes;
  d.smem_full = static_cast<uint32_t>(smem);
  if (job_lat && trace_capacity == 0) smem = align_up(engine_end, 16);  // drop the last part's histogram
  // keep >= 32: each warp's best list (keep+1 entries, rounded up to whole rows of 32) lives in shared
  // memory after the parts; smaller keep uses one register per lane
  if (job.keep >= 32) {
    d.big_len = static_cast<uint32_t>(align_up(job.keep + 1, 32));
    d.big_off = static_cast<uint32_t>(align_up(d.smem_full, 16));
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
    // random mode: a window of exactly two species draws the sites of its rarer species (Floyd's
    // sampling, see shuffle_part), starting from the window filled with the other species
    const bool floyd = !pj.systematic && !pj.chain && option(kOptBinaryFloyd) != 0;
    for (uint32_t w = 0; w < sl.n_windows; ++w) {
      const uint32_t word = floyd ? floyd_word(sl, w) : 0u;
      std::memcpy(base + P.win_off + 8ull * sl.n_windows + 4ull * w, &word, 4);
      if (word)
        for (uint32_t x = sl.windows[2 * w]; x < sl.windows[2 * w + 1]; ++x) base[P.species_off + x] = word >> 24;
    }
    const auto& k2d = k2_data[p];
    if (!k2d.first.empty()) std::memcpy(base + P.k2_off, k2d.first.data(), 4 * k2d.first.size());
    if (!k2d.second.empty()) std::memcpy(base + P.k2_shell_off, k2d.second.data(), 4 * k2d.second.size());
    if (!k2_nbp_data[p].empty())
      std::memcpy(base + P.k2_nbp_off, k2_nbp_data[p].data(), 4 * k2_nbp_data[p].size());
    if (d.lat) {
      const LatticeTables& LT = lat[p];
      std::memcpy(base + P.lat_site_off, LT.site_off.data(), 4 * LT.site_off.size());
      std::memcpy(base + P.lat_ent_off, LT.ent.data(), 4 * LT.ent.size());
      std::memcpy(base + P.lat_shell_off, LT.shell.data(), 4 * LT.shell.size());
      if (LT.words == 2) {
        std::memcpy(base + P.lat_tr_off, LT.tr.data(), sizeof(LatTrW<2>) * LT.tr.size());
      } else {  // one-word cell sets: the masks' first words only
        for (size_t k = 0; k < LT.tr.size(); ++k) {
          const LatTr& t = LT.tr[k];
          const LatTrW<1> o{t.sx, t.sxr, t.sy, t.syr, t.sz, t.szr, 0u, 0u, {t.mxh[0]}, {t.myh[0]}};
          std::memcpy(base + P.lat_tr_off + k * sizeof(LatTrW<1>), &o, sizeof(o));
        }
      }
      std::memcpy(base + P.lat_deg_off, LT.deg.data(), 4 * LT.deg.size());
    }
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
  if (pj.chain) {  // reference-stream mode: up to kBlock consecutive blocks per tile, one per thread
    const JobDesc& d = pj.desc;
    if (pj.total == 0) return;
    for (uint64_t b = 0; b < d.chain_blocks; b += kBlock) {
      Tile t{};
      t.job = job_index;
      t.start = b;
      t.count = std::min<uint64_t>(kBlock, d.chain_blocks - b);
      const uint64_t e = b + t.count;
      const auto start = [&](uint64_t x) { return x * d.chain_block + std::min(x, d.chain_rem); };
      t.chain_configs = (e == d.chain_blocks ? pj.total : start(e)) - start(b);
      tiles.push_back(t);
    }
    return;
  }
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
