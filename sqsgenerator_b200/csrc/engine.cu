// Host driver and C ABI of the SQS engine: validates a job, lays out its device blob, cuts it into
// tiles, launches the persistent kernel, watches progress/cancellation, and turns the candidate
// records into the reference's result set.
//
// Replaces sqsgen::run_optimization / optimizer<T,IMode,SMode>::run (include/sqsgen/sqs.h:299-634
// of dgehringer/sqsgenerator 0.5.6). The result set follows include/sqsgen/core/results.h:42-99:
// distinct configurations keyed by exact objective; see select_results() for the precise rule.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <exception>
#include <thread>
#include <unordered_set>
#include <vector>

#include "attr_tracker.h"
#include "host_copy.h"
#include "kernels.h"
#include "permutation.h"
#include "prepare.h"
#include "select.h"
#include "sqsg_internal.h"
#include "tiles.h"

namespace sqsg {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

// ------------------------------------------------------------------------------------------------
// Process-wide options
static std::atomic<long long> g_options[kOptCount] = {{0}, {static_cast<long long>(kWaitNs)}, {0}, {1},
                                                      {1ll << 20}, {4ll << 30}, {0}, {4}, {1}};
static const char* const kOptionNames[kOptCount] = {"force_general", "stage_wait_ns", "debug_skip_staging",
                                                    "use_tuning", "default_candidates", "rerun_record_bytes",
                                                    "rapidrand", "server_finalizers", "binary_floyd"};

long long option(Option o) { return g_options[o].load(std::memory_order_relaxed); }

static int option_index(const char* name) {
  if (!name) return -1;
  for (int k = 0; k < kOptCount; ++k)
    if (std::strcmp(name, kOptionNames[k]) == 0) return k;
  return -1;
}

static DynamicSmemTracker& smem_tracker() {
  static auto* t = new DynamicSmemTracker();  // never destroyed: used until exit
  return *t;
}

int raise_dynamic_smem(const void* kernel, size_t bytes) {
  int dev = 0;
  const cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return static_cast<int>(e);
  return smem_tracker().raise(dev, kernel, bytes, [&](size_t b) {
    return static_cast<int>(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 static_cast<int>(b)));
  });
}

#define CUDA_CHECK(expr)                                                                              \
  do {                                                                                                \
    cudaError_t err__ = (expr);                                                                       \
    if (err__ != cudaSuccess)                                                                         \
      throw cuda_error(std::string(#expr) + ": " + cudaGetErrorString(err__));                       \
  } while (0)

// ------------------------------------------------------------------------------------------------
// Device workspaces: grow-only buffers and streams, pooled per device.
struct DevBuf {
  void* p = nullptr;
  size_t size = 0;
  void ensure(size_t n) {
    if (n <= size) return;
    if (p) cudaFree(p);
    p = nullptr;
    size = 0;
    CUDA_CHECK(cudaMalloc(&p, n));
    size = n;
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

struct Workspace {
  int device = 0;
  cudaStream_t stream = nullptr, monitor = nullptr;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  DevBuf blob, records, counters, levels, tiles, jobs, queue, status, trace_sp, trace_bd, trace_obj, trace_id;
  SelectScratch select;
  // Cancellation flag in device memory (CTAs read it once per tile from L2; a flag in mapped host
  // memory cost a PCIe round trip per tile, queued across hundreds of CTAs), raised by a copy on
  // the monitor stream from a pinned word holding 1.
  int32_t* cancel_dev = nullptr;
  int32_t* one_host = nullptr;
  explicit Workspace(int dev) : device(dev) {
    CUDA_CHECK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CUDA_CHECK(cudaStreamCreateWithFlags(&monitor, cudaStreamNonBlocking));
    CUDA_CHECK(cudaEventCreate(&ev_start));
    CUDA_CHECK(cudaEventCreate(&ev_stop));
    CUDA_CHECK(cudaMalloc(reinterpret_cast<void**>(&cancel_dev), 256));
    CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&one_host), 64, cudaHostAllocDefault));
    one_host[0] = 1;
  }
  ~Workspace() {
    select.release();
    if (stream) cudaStreamDestroy(stream);
    if (monitor) cudaStreamDestroy(monitor);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_stop) cudaEventDestroy(ev_stop);
    if (cancel_dev) cudaFree(cancel_dev);
    if (one_host) cudaFreeHost(one_host);
  }
};

class WorkspacePool {
 public:
  std::unique_ptr<Workspace> acquire(int device) {
    {
      std::lock_guard<std::mutex> l(m_);
      auto& v = free_[device];
      if (!v.empty()) {
        auto w = std::move(v.back());
        v.pop_back();
        return w;
      }
    }
    return std::make_unique<Workspace>(device);
  }
  void release(std::unique_ptr<Workspace> w) {
    std::lock_guard<std::mutex> l(m_);
    free_[w->device].push_back(std::move(w));
  }

 private:
  std::mutex m_;
  std::map<int, std::vector<std::unique_ptr<Workspace>>> free_;
};

static WorkspacePool& pool() {
  static auto* p = new WorkspacePool();  // never destroyed: avoids CUDA calls during exit
  return *p;
}

struct WorkspaceLease {
  std::unique_ptr<Workspace> w;
  explicit WorkspaceLease(int device) : w(pool().acquire(device)) {}
  ~WorkspaceLease() {
    if (w) pool().release(std::move(w));
  }
  Workspace* operator->() { return w.get(); }
};

static int device_sm_count(int dev) {
  int n = 0;
  CUDA_CHECK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  return n;
}

// The dynamic shared-memory attribute is per device: it is raised on the current device (every
// caller has made the job's device current).
static void configure_kernel(size_t smem) {
  for (int kind = 0; kind < kKindCount; ++kind) {
    const int err = raise_dynamic_smem(reinterpret_cast<const void*>(kernel_of(kind)), smem);
    if (err != 0)
      throw cuda_error(std::string("cudaFuncSetAttribute(MaxDynamicSharedMemorySize): ") +
                       cudaGetErrorString(static_cast<cudaError_t>(err)));
  }
}

static uint32_t launch_grid(int dev, size_t smem, size_t n_tiles, EngineKernel kernel, uint32_t ctas = 0) {
  configure_kernel(smem);
  int per_sm = 0;
  CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, smem));
  if (per_sm <= 0) throw unsupported_error("the job needs more shared memory than one SM offers");
  if (ctas > 0) per_sm = std::min<int>(per_sm, static_cast<int>(ctas));
  size_t grid = static_cast<size_t>(per_sm) * device_sm_count(dev);
  return static_cast<uint32_t>(std::max<size_t>(1, std::min(grid, n_tiles)));
}

static size_t max_dynamic_smem(int dev) {
  int v = 0;
  CUDA_CHECK(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  size_t stat = 0;
  for (int kind = 0; kind < kKindCount; ++kind) {
    cudaFuncAttributes a{};
    CUDA_CHECK(cudaFuncGetAttributes(&a, kernel_of(kind)));
    stat = std::max<size_t>(stat, a.sharedSizeBytes);
  }
  return static_cast<size_t>(v) - stat;
}

// ------------------------------------------------------------------------------------------------
// Results
template <class T> static T read_t(const uint8_t* p) {
  T v;
  std::memcpy(&v, p, sizeof(T));
  return v;
}

struct Run {
  int prec = 1;
  uint32_t n_parts = 1;
  std::vector<PartMeta> parts;
  size_t tsz = 8;
  uint64_t count = 0;
  ByteVec objective, sub_objective, sro;  // raw T bytes
  ByteVec species;
  IdVec id;
  sqsg_statistics stats{};
  // keep+1 best distinct objectives with evaluation counts and id checksums (exact unless
  // levels_exact is false), and whether the record set was cut at the capacity.
  std::vector<double> level_value;
  std::vector<uint64_t> level_count, level_checksum;
  bool truncated = false, levels_exact = true;
  uint64_t candidates = 0;
  uint64_t h2d_bytes = 0, d2h_bytes = 0;
  uint64_t stage_ns[SQSG_STAGE_COUNT] = {};  // host-side time per stage of the call (sqsg_run_stages)
};

// The reference accepts a configuration when its objective is <= the search threshold, which only
// ever falls to nth_best(keep) — the (keep+1)-th best distinct objective in the collection
// (sqs.h:421-438, results.h:78-82) — and never evicts. Every configuration at or below the final
// (keep+1)-th best distinct objective T* is therefore in the reference's result set on every run;
// entries above T* depend on thread timing. The result set here is exactly the deterministic part:
// all distinct configurations with objective <= T* (T* = +inf with fewer distinct objectives),
// sorted by objective then id, at most max_results_per_objective+1 per objective (sqs.h:423-426
// admits one more than the cap).
template <class T>
static void select_results(const PreparedJob& pj, const std::vector<uint8_t>& recs, uint64_t n, Run& run,
                           bool have_tstar, double tstar_levels) {
  const size_t rb = pj.record_bytes;
  struct Key {
    T obj;
    uint64_t id;
    uint64_t idx;
  };
  std::vector<Key> keys(n);
  for (uint64_t i = 0; i < n; ++i) keys[i] = Key{read_t<T>(&recs[i * rb]), read_t<uint64_t>(&recs[i * rb + 8]), i};
  T tstar = std::numeric_limits<T>::infinity();
  if (have_tstar) {
    tstar = static_cast<T>(tstar_levels);
    keys.erase(std::remove_if(keys.begin(), keys.end(), [&](const Key& k) { return !(k.obj <= tstar); }), keys.end());
  }
  std::sort(keys.begin(), keys.end(), [](const Key& a, const Key& b) {
    if (a.obj != b.obj) return a.obj < b.obj;
    return a.id < b.id;
  });
  if (!have_tstar) {
    uint64_t distinct = 0;
    for (size_t k = 0; k < keys.size(); ++k)
      if (k == 0 || keys[k].obj != keys[k - 1].obj) {
        if (distinct == pj.keep) {
          tstar = keys[k].obj;
          break;
        }
        ++distinct;
      }
  }
  const JobDesc& d = pj.desc;
  size_t sp_total = 0, skk_total = 0;
  for (auto& p : pj.parts) {
    sp_total += p.N;
    skk_total += static_cast<size_t>(p.S) * p.K * p.K;
  }
  size_t end = 0;
  while (end < keys.size() && keys[end].obj <= tstar) ++end;
  // Systematic ranks are unique, so only random runs can return one configuration twice. Equal
  // configurations have equal objectives, so duplicates are removed inside each objective group:
  // the group is ordered by (species hash, id) and, among records with equal species, the one with
  // the smallest id stays (the first one met in (objective, id) order).
  const bool dedup = !pj.systematic;
  std::vector<uint8_t> keep_rec(end, 1);
  if (dedup) {
    auto species_eq = [&](uint64_t x, uint64_t y) {
      for (uint32_t p = 0; p < d.n_parts; ++p) {
        const size_t off = d.parts[p].rec_species_off;
        if (std::memcmp(&recs[x * rb + off], &recs[y * rb + off], d.parts[p].n_sites) != 0) return false;
      }
      return true;
    };
    std::vector<std::pair<uint64_t, size_t>> grp;  // (species hash, position in keys)
    for (size_t g0 = 0; g0 < end;) {
      size_t g1 = g0 + 1;
      while (g1 < end && keys[g1].obj == keys[g0].obj) ++g1;
      if (g1 - g0 > 1) {
        grp.clear();
        for (size_t k = g0; k < g1; ++k) {
          uint64_t h = 0xcbf29ce484222325ull;  // FNV-1a over the record's species bytes
          const uint8_t* r = &recs[keys[k].idx * rb];
          for (uint32_t p = 0; p < d.n_parts; ++p)
            for (uint32_t x = 0; x < d.parts[p].n_sites; ++x) h = (h ^ r[d.parts[p].rec_species_off + x]) * 0x100000001b3ull;
          grp.emplace_back(h, k);
        }
        std::sort(grp.begin(), grp.end());  // ties in hash keep (objective, id) order via the position
        for (size_t u = 0; u < grp.size();) {
          size_t v = u + 1;
          while (v < grp.size() && grp[v].first == grp[u].first) ++v;
          for (size_t x = u + 1; x < v; ++x)
            for (size_t y = u; y < x; ++y)
              if (keep_rec[grp[y].second] && species_eq(keys[grp[x].second].idx, keys[grp[y].second].idx)) {
                keep_rec[grp[x].second] = 0;
                break;
              }
          u = v;
        }
      }
      g0 = g1;
    }
  }
  run.objective.reserve(end * sizeof(T));
  run.species.reserve(end * sp_total);
  run.sro.reserve(end * skk_total * sizeof(T));
  T cur_obj = T(0);
  bool have_cur = false;
  uint64_t cur_count = 0;
  for (size_t k = 0; k < end; ++k) {
    if (!keep_rec[k]) continue;
    const Key& key = keys[k];
    const uint8_t* r = &recs[key.idx * rb];
    if (!have_cur || key.obj != cur_obj) {
      cur_obj = key.obj;
      have_cur = true;
      cur_count = 0;
    }
    if (pj.max_rpo >= 0 && cur_count > static_cast<uint64_t>(pj.max_rpo)) continue;
    ++cur_count;
    run.objective.insert(run.objective.end(), r, r + sizeof(T));
    for (uint32_t p = 0; p < d.n_parts; ++p) {
      const PartDesc& P = d.parts[p];
      run.sub_objective.insert(run.sub_objective.end(), r + P.rec_obj_off, r + P.rec_obj_off + sizeof(T));
      run.species.insert(run.species.end(), r + P.rec_species_off, r + P.rec_species_off + P.n_sites);
      const size_t skk = static_cast<size_t>(P.n_shells) * P.n_species * P.n_species;
      run.sro.insert(run.sro.end(), r + P.rec_sro_off, r + P.rec_sro_off + skk * sizeof(T));
    }
    run.id.push_back(key.id);
    run.count++;
  }
}

// Candidate sets at least this large are selected on the device.
constexpr uint64_t kDeviceSelectMin = 32768;
// Candidate capacity of a job that leaves max_results at 0 (option "default_candidates", 2^20 = 16 MiB
// of candidates by default; a job whose buffer overflows runs again with a buffer sized from its
// exact level counts, within rerun_limit).
static uint64_t default_candidates() { return static_cast<uint64_t>(option(kOptDefaultCandidates)); }
// Size of the full records (rebuilt on the device and copied out) that a re-run may produce when the
// first pass overflowed its candidate buffer (option "rerun_record_bytes", 4 GiB by default). Random
// runs over small configuration spaces revisit configurations; their re-run keeps each distinct one
// once when its keys are exact. A job whose result set is larger keeps the records of its first pass
// (truncated; the objective levels stay exact).
static uint64_t rerun_limit(const PreparedJob& pj) {
  return static_cast<uint64_t>(option(kOptRerunRecordBytes)) / pj.record_bytes;
}

// Lattice path: 64-bit AND-popcount units per configuration of part p (translation classes from the
// part's shell table {first class, first self-reverse class, end, pairs} x species pairs a <= b < K-1
// x words per cell set).
static uint64_t lattice_units(const PreparedJob& pj, uint32_t p) {
  const PartDesc& P = pj.desc.parts[p];
  const uint64_t na = P.n_species - 1;
  uint64_t classes = 0;
  for (uint32_t sh = 0; sh < P.n_shells; ++sh) {
    uint32_t e[4];
    std::memcpy(e, pj.blob.data() + P.blob_off + P.lat_shell_off + 16 * sh, 16);
    classes += e[2] - e[0];
  }
  return classes * na * (na + 1) / 2 * pj.desc.lat_words;  // one unit per 64-bit word of a cell set
}

// Estimated cost of one configuration in pair evaluations of the pair-stream path (its unit of
// work), from B200 measurements: the pair stream costs one per pair, the lattice path about one per
// AND-popcount unit, the bit-mask path about an eighth per pair; shuffling and setting up a
// configuration cost about two per site on every path. The served form sizes tiles and divides the
// SMs between its rings by it.
static double config_cost(const PreparedJob& pj) {
  double cost = 0.0;
  for (uint32_t p = 0; p < pj.desc.n_parts; ++p) {
    const PartDesc& P = pj.desc.parts[p];
    const double sites = static_cast<double>(P.n_sites);
    const double pairs = static_cast<double>(pj.parts[p].P);
    if (pj.desc.k2)
      cost += pairs / 8.0 + sites;
    else if (pj.desc.lat)
      cost += static_cast<double>(lattice_units(pj, p)) + 2.0 * sites;
    else
      cost += pairs + 2.0 * sites;
  }
  return std::max(1.0, cost);
}

static RecordLayout record_layout(const PreparedJob& pj) {
  RecordLayout L;
  L.record_bytes = static_cast<uint32_t>(pj.record_bytes);
  L.tsz = static_cast<uint32_t>(pj.tsz);
  L.n_parts = pj.desc.n_parts;
  for (uint32_t p = 0; p < pj.desc.n_parts; ++p) {
    const PartDesc& P = pj.desc.parts[p];
    L.obj_off[p] = P.rec_obj_off;
    L.species_off[p] = P.rec_species_off;
    L.n_sites[p] = P.n_sites;
    L.sro_off[p] = P.rec_sro_off;
    L.sro_bytes[p] = static_cast<uint32_t>(static_cast<size_t>(P.n_shells) * P.n_species * P.n_species * pj.tsz);
  }
  return L;
}

// What one pass of a job left behind: its exact objective levels (keep+1 smallest distinct
// objectives with evaluation counts and id checksums) and the final threshold T*, or a request to
// run the job again.
//  - The device level table is exact unless it ran out of slots (many distinct objectives while
//    the threshold was still high). Then, if the record buffer held every candidate, the levels are
//    rebuilt from the records: every evaluation at or below the threshold of its time — so every
//    evaluation at or below T* — is a record.
//  - A record buffer that overflowed asks for a re-run (same tiles, same seeds and ids, same
//    evaluations) whose threshold starts at T* (exact levels: the buffer is sized from their counts)
//    or at the (keep+1)-th distinct objective of the stored records, an upper bound of T*.
//  - When the evaluations at or below T* are too many for any buffer but the random job's
//    configurations have exact keys, the re-run stores each distinct configuration once (with its
//    smallest id) in a table sized from min(evaluations, arrangements): in random mode repeats make
//    up most of a small configuration space.
struct Outcome {
  bool rerun = false;
  uint64_t rerun_capacity = 0;
  uint64_t rerun_slots = 0;  // > 0: a deduplicating re-run with a table of this many slots
  double rerun_threshold = 0.0;
  bool levels_exact = false;
  double tstar = std::numeric_limits<double>::infinity();
  std::vector<double> value;
  std::vector<uint64_t> count, checksum;
};

static void levels_from_records(const PreparedJob& pj, const std::vector<Cand>& recs, uint64_t n, Outcome& o) {
  // the keep+1 smallest distinct keys, ascending: one pass that inserts only keys below the current
  // largest (rare once the array is full), then one pass that counts the records at those keys
  const size_t m = static_cast<size_t>(pj.keep) + 1;
  std::vector<unsigned long long> best;
  best.reserve(m + 1);
  for (uint64_t i = 0; i < n; ++i) {
    const unsigned long long key = ord_bits(recs[i].objective);
    if (best.size() == m && key >= best.back()) continue;
    const auto it = std::lower_bound(best.begin(), best.end(), key);
    if (it != best.end() && *it == key) continue;
    best.insert(it, key);
    if (best.size() > m) best.pop_back();
  }
  std::vector<uint64_t> count(best.size(), 0);
  std::vector<uint32_t> sa(best.size(), 0), sb(best.size(), 0);
  for (uint64_t i = 0; i < n && !best.empty(); ++i) {
    const unsigned long long key = ord_bits(recs[i].objective);
    if (key > best.back()) continue;
    const size_t k = static_cast<size_t>(std::lower_bound(best.begin(), best.end(), key) - best.begin());
    const unsigned long long h = mix64(recs[i].id);
    count[k]++;
    sa[k] += static_cast<uint32_t>(h);
    sb[k] += static_cast<uint32_t>(h >> 32);
  }
  for (size_t k = 0; k < best.size(); ++k) {
    o.value.push_back(from_ord(best[k]));
    o.count.push_back(count[k]);
    o.checksum.push_back(static_cast<uint64_t>(sa[k]) | (static_cast<uint64_t>(sb[k]) << 32));
  }
}

static Outcome assess(const PreparedJob& pj, const unsigned long long* cnt, const LevelSlot* lv,
                      const std::vector<Cand>& recs, uint64_t stored, uint64_t capacity, bool may_rerun,
                      uint64_t max_capacity) {
  Outcome o;
  const bool full = cnt[kRecordsFull] != 0 || cnt[kCandidates] > capacity;
  const bool overflow = cnt[kLevelOverflow] != 0;
  if (!overflow) {
    std::vector<LevelSlot> used;
    for (int k = 0; k < kLevelSlots; ++k)
      if (lv[k].key) used.push_back(lv[k]);
    std::sort(used.begin(), used.end(), [](const LevelSlot& a, const LevelSlot& b) { return a.key < b.key; });
    uint64_t need = 0;
    for (size_t k = 0; k < used.size() && k <= pj.keep; ++k) {
      o.value.push_back(from_ord(used[k].key));
      o.count.push_back(used[k].count);
      o.checksum.push_back(static_cast<uint64_t>(used[k].sum_a) | (static_cast<uint64_t>(used[k].sum_b) << 32));
      need += used[k].count;
    }
    o.levels_exact = true;
    if (used.size() > pj.keep) o.tstar = from_ord(used[pj.keep].key);
    if (full && may_rerun && need + 64 <= max_capacity) {
      o.rerun = true;
      o.rerun_capacity = std::max<uint64_t>(need + 64, 1024);
      o.rerun_threshold = o.tstar;
    } else if (full && may_rerun && pj.dedup_ok) {
      const uint64_t distinct = std::min<uint64_t>(need, pj.dedup_space);
      uint64_t slots = 1024;
      while (slots < 2 * distinct) slots <<= 1;  // load factor at most 1/2
      if (distinct + 64 + slots * sizeof(DedupSlot) / sizeof(Cand) <= max_capacity) {
        o.rerun = true;
        o.rerun_capacity = std::max<uint64_t>(distinct + 64, 1024);
        o.rerun_slots = slots;
        o.rerun_threshold = o.tstar;
      }
    }
    return o;
  }
  levels_from_records(pj, recs, stored, o);
  if (!full) {
    o.levels_exact = true;
    if (o.value.size() > pj.keep) o.tstar = o.value[pj.keep];
    return o;
  }
  // neither the table nor the records are complete
  if (may_rerun && o.value.size() > pj.keep) {
    o.rerun = true;
    o.rerun_capacity = std::min<uint64_t>(max_capacity, std::max<uint64_t>(capacity * 2, 1024));
    o.rerun_threshold = o.value[pj.keep];
  }
  return o;
}

// The result set of a finished job's n device-resident candidates. Large sets with exact levels are
// selected on the device (select_on_device); otherwise the candidates are filtered (objective <= T*)
// and ordered (objective, id) on the host, systematic runs are capped per objective, the selected
// candidates' full records are rebuilt on the device (sqsg_materialize) and select_results removes
// repeats and applies the cap. `host_cands` may hold the candidates already downloaded.
static void finish_selection(SelectScratch& scratch, cudaStream_t stream, const PreparedJob& pj, const JobDesc& dev_desc,
                             const Cand* d_cands, uint64_t n, std::vector<Cand>& host_cands, const Outcome& o,
                             bool table_exact, Run& run, uint64_t& d2h_bytes) {
  Materializer mat;
  mat.job = dev_desc;
  mat.smem = pj.desc.smem_full;
  if (n >= kDeviceSelectMin && table_exact && o.levels_exact) {
    SelectedSet set;
    if (select_on_device(scratch, stream, record_layout(pj), d_cands, n, o.value, !pj.systematic, pj.max_rpo,
                         pj.range_first + pj.range_count + 1, mat, set)) {
      run.count = set.count;
      run.objective = std::move(set.objective);
      run.sub_objective = std::move(set.sub_objective);
      run.species = std::move(set.species);
      run.sro = std::move(set.sro);
      run.id = std::move(set.id);
      d2h_bytes += run.objective.size() + run.sub_objective.size() + run.species.size() + run.sro.size() +
                   run.id.size() * 8;
      return;
    }
  }
  if (host_cands.size() != n) {
    host_cands.resize(n);
    if (n) CUDA_CHECK(cudaMemcpyAsync(host_cands.data(), d_cands, n * sizeof(Cand), cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    d2h_bytes += n * sizeof(Cand);
  }
  // keep+1 best distinct objectives among the stored candidates when the levels are not exact
  double tstar = o.tstar;
  if (!o.levels_exact) {
    std::vector<double> v;
    v.reserve(n);
    for (auto& c : host_cands) v.push_back(c.objective);
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    tstar = v.size() > pj.keep ? v[pj.keep] : std::numeric_limits<double>::infinity();
  }
  std::vector<Cand> sel;
  for (auto& c : host_cands)
    if (c.objective <= tstar) sel.push_back(c);
  std::sort(sel.begin(), sel.end(), [](const Cand& a, const Cand& b) {
    return a.objective != b.objective ? a.objective < b.objective : a.id < b.id;
  });
  if (pj.systematic && pj.max_rpo >= 0) {  // ranks are unique: the cap applies before rebuilding
    std::vector<Cand> capped;
    uint64_t cur = 0;
    for (size_t k = 0; k < sel.size(); ++k) {
      cur = (k == 0 || sel[k].objective != sel[k - 1].objective) ? 0 : cur + 1;
      if (cur <= static_cast<uint64_t>(pj.max_rpo)) capped.push_back(sel[k]);
    }
    sel.swap(capped);
  }
  const uint64_t m = sel.size();
  std::vector<uint8_t> recs(m * pj.record_bytes);
  if (m) {
    if (scratch.stream != stream) {
      scratch.release();
      scratch.stream = stream;
    }
    auto* d_sel = static_cast<Cand*>(scratch.get(7, m * sizeof(Cand)));
    auto* d_recs = static_cast<uint8_t*>(scratch.get(19, m * pj.record_bytes));
    CUDA_CHECK(cudaMemcpyAsync(d_sel, sel.data(), m * sizeof(Cand), cudaMemcpyHostToDevice, stream));
    if (materialize(scratch, stream, mat, d_sel, static_cast<uint32_t>(m), d_recs) != 0)
      throw cuda_error("internal error: a rebuilt record's objective differs from the engine's");
    CUDA_CHECK(cudaMemcpyAsync(recs.data(), d_recs, recs.size(), cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    d2h_bytes += recs.size();
  }
  if (pj.prec == 1)
    select_results<double>(pj, recs, m, run, true, tstar);
  else
    select_results<float>(pj, recs, m, run, true, tstar);
}

// ------------------------------------------------------------------------------------------------
// Executing prepared jobs on one device.
struct TraceOut {
  uint64_t capacity = 0;
  uint64_t* count = nullptr;
  uint8_t* species = nullptr;
  uint32_t* bonds = nullptr;
  void* objective = nullptr;
  uint64_t* id = nullptr;
};

static uint64_t now_ns() {
  return static_cast<uint64_t>(
      std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
          .count());
}

// Runs a set of prepared jobs in one persistent launch (one job = the plain path). Returns once
// every job finished, was cancelled, or a device error was raised.
static void execute(std::vector<PreparedJob>& pjs, const std::vector<const sqsg_job*>& srcs, int device,
                    std::vector<Run>& runs, const TraceOut* trace) {
  const uint64_t t0 = now_ns();
  CUDA_CHECK(cudaSetDevice(device));
  WorkspaceLease ws(device);
  const size_t nj = pjs.size();
  const size_t smem_limit = max_dynamic_smem(device);
  size_t smem = 0, blob_total = 0;
  std::vector<size_t> blob_off(nj), rec_off(nj);
  std::vector<uint64_t> capacity(nj), slots(nj, 0);
  std::vector<double> start_threshold(nj, 0.0);
  std::vector<bool> fixed_threshold(nj, false);
  size_t rec_total = 0;
  for (size_t j = 0; j < nj; ++j) {
    if (pjs[j].desc.smem_bytes > smem_limit)
      throw unsupported_error("the job needs " + std::to_string(pjs[j].desc.smem_bytes) +
                              " bytes of shared memory per CTA; this device offers " + std::to_string(smem_limit));
    smem = std::max<size_t>(smem, pjs[j].desc.smem_bytes);
    blob_off[j] = blob_total;
    blob_total = align_up(blob_total + pjs[j].blob.size(), 256);
    capacity[j] = pjs[j].max_results ? pjs[j].max_results : default_candidates();
    if (pjs[j].rerun_capacity) {
      capacity[j] = pjs[j].rerun_capacity;
      slots[j] = pjs[j].rerun_slots;
      fixed_threshold[j] = true;
      start_threshold[j] = pjs[j].rerun_threshold;
    }
  }
  std::vector<Tile> tiles;
  for (size_t j = 0; j < nj; ++j)
    make_tiles(pjs[j], static_cast<uint32_t>(j), tiles, pjs[j].tuning.tile_cap ? pjs[j].tuning.tile_cap : 1u << 16);

  const uint64_t t_setup = now_ns();
  float loop_ms_total = 0.f;
  for (int attempt = 0; attempt < 4; ++attempt) {
    rec_total = 0;
    for (size_t j = 0; j < nj; ++j) {  // candidates, then the distinct-configuration table (if any)
      rec_off[j] = rec_total;
      rec_total = align_up(align_up(rec_total + capacity[j] * sizeof(Cand), 256) + slots[j] * sizeof(DedupSlot), 256);
    }
    ws->blob.ensure(std::max<size_t>(blob_total, 256));
    ws->records.ensure(std::max<size_t>(rec_total, 256));
    ws->counters.ensure(nj * kNumCounters * sizeof(unsigned long long));
    ws->levels.ensure(nj * kLevelSlots * sizeof(LevelSlot));
    ws->tiles.ensure(std::max<size_t>(tiles.size(), 1) * sizeof(Tile));
    ws->jobs.ensure(nj * sizeof(JobDesc));
    ws->queue.ensure(sizeof(QueueCtl));
    ws->status.ensure(sizeof(unsigned long long));
    auto* counters = static_cast<unsigned long long*>(ws->counters.p);
    std::vector<unsigned long long> init(nj * kNumCounters, 0);
    std::vector<JobDesc> descs(nj);
    for (size_t j = 0; j < nj; ++j) {
      JobDesc d = pjs[j].desc;
      d.blob = static_cast<const uint8_t*>(ws->blob.p) + blob_off[j];
      d.records = static_cast<uint8_t*>(ws->records.p) + rec_off[j];
      d.capacity = capacity[j];
      if (slots[j]) {
        d.dedup = reinterpret_cast<DedupSlot*>(static_cast<uint8_t*>(ws->records.p) +
                                               align_up(rec_off[j] + capacity[j] * sizeof(Cand), 256));
        d.dedup_mask = slots[j] - 1;
        CUDA_CHECK(cudaMemsetAsync(d.dedup, 0xff, slots[j] * sizeof(DedupSlot), ws->stream));
      }
      d.counters = counters + j * kNumCounters;
      d.levels = static_cast<LevelSlot*>(ws->levels.p) + j * kLevelSlots;
      const double maxv = pjs[j].prec == 1 ? std::numeric_limits<double>::max()
                                           : static_cast<double>(std::numeric_limits<float>::max());
      init[j * kNumCounters + kThreshold] = ord_bits(fixed_threshold[j] ? start_threshold[j] : maxv);
      init[j * kNumCounters + kBest] = ord_bits(std::numeric_limits<double>::infinity());
      if (trace && trace->capacity) {
        const size_t sp = d.trace_species_stride, bd = d.trace_bonds_stride;
        ws->trace_sp.ensure(std::max<size_t>(trace->capacity * sp, 16));
        ws->trace_bd.ensure(std::max<size_t>(trace->capacity * bd * 4, 16));
        ws->trace_obj.ensure(std::max<size_t>(trace->capacity * pjs[j].tsz, 16));
        ws->trace_id.ensure(std::max<size_t>(trace->capacity * 8, 16));
        d.trace_species = static_cast<uint8_t*>(ws->trace_sp.p);
        d.trace_bonds = static_cast<uint32_t*>(ws->trace_bd.p);
        d.trace_obj = ws->trace_obj.p;
        d.trace_id = static_cast<uint64_t*>(ws->trace_id.p);
      }
      descs[j] = d;
      CUDA_CHECK(cudaMemcpyAsync(static_cast<uint8_t*>(ws->blob.p) + blob_off[j], pjs[j].blob.data(),
                                 pjs[j].blob.size(), cudaMemcpyHostToDevice, ws->stream));
    }
    CUDA_CHECK(cudaMemcpyAsync(counters, init.data(), init.size() * sizeof(unsigned long long),
                               cudaMemcpyHostToDevice, ws->stream));
    CUDA_CHECK(cudaMemcpyAsync(ws->jobs.p, descs.data(), nj * sizeof(JobDesc), cudaMemcpyHostToDevice, ws->stream));
    if (!tiles.empty())
      CUDA_CHECK(cudaMemcpyAsync(ws->tiles.p, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice,
                                 ws->stream));
    uint64_t h2d_bytes = init.size() * sizeof(unsigned long long) + nj * sizeof(JobDesc) + tiles.size() * sizeof(Tile);
    for (size_t j = 0; j < nj; ++j) h2d_bytes += pjs[j].blob.size();
    CUDA_CHECK(cudaMemsetAsync(ws->levels.p, 0, nj * kLevelSlots * sizeof(LevelSlot), ws->stream));
    CUDA_CHECK(cudaMemsetAsync(ws->queue.p, 0, sizeof(QueueCtl), ws->stream));
    CUDA_CHECK(cudaMemsetAsync(ws->status.p, 0, sizeof(unsigned long long), ws->stream));
    CUDA_CHECK(cudaMemsetAsync(ws->cancel_dev, 0, sizeof(int32_t), ws->stream));
    bool cancel_sent = false;

    // one kernel per launch: the jobs of a launch are of one kind, except that bit-mask jobs may share a
    // launch of the general path (their columns and stream exist too); lattice jobs never mix
    int kind = kind_of(pjs[0].desc);
    for (size_t j = 1; j < nj; ++j) {
      const int kj = kind_of(pjs[j].desc);
      if (kj == kind) continue;
      if (is_lattice_kind(kj) && is_lattice_kind(kind) && kj != kKindLatW && kind != kKindLatW) {
        kind = kKindLat;  // the eight-species kernel holds every one-word variant
        continue;
      }
      if (is_lattice_kind(kj) || is_lattice_kind(kind))
        throw std::logic_error("lattice jobs mixed with others in one launch");
      kind = kKindWide;
    }
    const EngineKernel kernel = kernel_of(kind);
    const uint32_t grid = launch_grid(device, smem, tiles.size(), kernel, nj == 1 ? pjs[0].tuning.ctas : 0u);
    const uint64_t t_launch = now_ns();
    CUDA_CHECK(cudaEventRecord(ws->ev_start, ws->stream));
    if (!tiles.empty()) {
      kernel<<<grid, kBlock, smem, ws->stream>>>(
          static_cast<const JobDesc*>(ws->jobs.p), static_cast<const Tile*>(ws->tiles.p),
          static_cast<uint32_t>(tiles.size()), static_cast<QueueCtl*>(ws->queue.p), ws->cancel_dev,
          static_cast<unsigned long long*>(ws->status.p), nullptr);
      CUDA_CHECK(cudaGetLastError());
    }
    CUDA_CHECK(cudaEventRecord(ws->ev_stop, ws->stream));

    // Watch progress: cancellation flags and progress callbacks are served from this thread.
    std::vector<uint64_t> next_cb(nj, 0);
    for (size_t j = 0; j < nj; ++j) {
      const uint64_t chunk = srcs[j]->chunk_size ? srcs[j]->chunk_size : 100000;
      next_cb[j] = chunk;
    }
    std::vector<unsigned long long> mirror;
    bool any_watch = false;
    for (size_t j = 0; j < nj; ++j) any_watch |= srcs[j]->cancel != nullptr || srcs[j]->callback != nullptr;
    while (true) {
      cudaError_t q = cudaEventQuery(ws->ev_stop);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) CUDA_CHECK(q);
      if (!any_watch) {
        CUDA_CHECK(cudaEventSynchronize(ws->ev_stop));
        break;
      }
      std::this_thread::sleep_for(std::chrono::microseconds(500));
      bool stop = false;
      for (size_t j = 0; j < nj; ++j)
        if (srcs[j]->cancel && *srcs[j]->cancel) stop = true;
      bool need_cb = false;
      for (size_t j = 0; j < nj; ++j) need_cb |= srcs[j]->callback != nullptr;
      if (need_cb) {
        mirror.resize(nj * kNumCounters);
        CUDA_CHECK(cudaMemcpyAsync(mirror.data(), counters, nj * kNumCounters * sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost, ws->monitor));
        CUDA_CHECK(cudaStreamSynchronize(ws->monitor));
        for (size_t j = 0; j < nj; ++j) {
          if (!srcs[j]->callback) continue;
          const uint64_t fin = mirror[j * kNumCounters + kFinished];
          if (fin < next_cb[j]) continue;
          const uint64_t chunk = srcs[j]->chunk_size ? srcs[j]->chunk_size : 100000;
          while (next_cb[j] <= fin) next_cb[j] += chunk;
          sqsg_statistics st{};
          st.finished = fin;
          st.working = pjs[j].range_count > fin ? pjs[j].range_count - fin : 0;
          st.best_objective = from_ord(mirror[j * kNumCounters + kBest]);
          st.timings_ns[SQSG_TIMING_TOTAL] = now_ns() - t0;
          if (srcs[j]->callback(&st, srcs[j]->user) != 0) stop = true;
        }
      }
      if (stop && !cancel_sent) {
        CUDA_CHECK(cudaMemcpyAsync(ws->cancel_dev, ws->one_host, sizeof(int32_t), cudaMemcpyHostToDevice,
                                   ws->monitor));
        cancel_sent = true;
      }
    }
    CUDA_CHECK(cudaGetLastError());
    float ms = 0.f;
    CUDA_CHECK(cudaEventElapsedTime(&ms, ws->ev_start, ws->ev_stop));
    loop_ms_total += ms;
    const uint64_t t_done = now_ns();
    std::vector<unsigned long long> cnt(nj * kNumCounters);
    CUDA_CHECK(cudaMemcpy(cnt.data(), counters, cnt.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    unsigned long long status = 0;
    CUDA_CHECK(cudaMemcpy(&status, ws->status.p, sizeof(status), cudaMemcpyDeviceToHost));
    if (status == kErrStageTimeout) throw timeout_error("shared-memory staging wait timed out on the device");
    if (status != 0) throw cuda_error("device error code " + std::to_string(status));
    for (size_t j = 0; j < nj; ++j) check_job_counters(cnt.data() + j * kNumCounters);
    // deduplicating re-runs: the table's distinct configurations become the job's candidates
    for (size_t j = 0; j < nj; ++j)
      if (slots[j])
        cnt[j * kNumCounters + kCandidates] =
            compact_dedup(ws->select, ws->stream, descs[j].dedup, slots[j],
                          reinterpret_cast<Cand*>(static_cast<uint8_t*>(ws->records.p) + rec_off[j]), capacity[j]);
    // Every job's counters and level table come back; a job whose record buffer overflowed is re-run
    // (see assess) when the caller left the capacity to the library. Records come back only when
    // the level table overflowed (the levels are then rebuilt from them on the host) or the set is
    // small; otherwise the result set is selected on the device and only it is copied out.
    bool rerun = false;
    std::vector<std::vector<Cand>> recs(nj);
    std::vector<Outcome> outc(nj);
    uint64_t d2h_bytes = cnt.size() * sizeof(unsigned long long) + 8;
    std::vector<LevelSlot> lv_all(nj * kLevelSlots);  // every job's level table in one copy
    CUDA_CHECK(cudaMemcpy(lv_all.data(), ws->levels.p, lv_all.size() * sizeof(LevelSlot), cudaMemcpyDeviceToHost));
    d2h_bytes += lv_all.size() * sizeof(LevelSlot);
    for (size_t j = 0; j < nj; ++j) {
      const unsigned long long* cj = &cnt[j * kNumCounters];
      const LevelSlot* lv = lv_all.data() + j * kLevelSlots;
      const uint64_t n = std::min<uint64_t>(cj[kCandidates], capacity[j]);
      if (cj[kLevelOverflow]) {
        recs[j].resize(n);
        if (n)
          CUDA_CHECK(cudaMemcpy(recs[j].data(), static_cast<uint8_t*>(ws->records.p) + rec_off[j], n * sizeof(Cand),
                                cudaMemcpyDeviceToHost));
        d2h_bytes += n * sizeof(Cand);
      }
      const bool may_rerun = !pjs[j].max_results && pjs[j].passes + attempt < 2;
      outc[j] = assess(pjs[j], cj, lv, recs[j], n, capacity[j], may_rerun, rerun_limit(pjs[j]));
      if (outc[j].rerun) {
        capacity[j] = outc[j].rerun_capacity;
        slots[j] = outc[j].rerun_slots;
        fixed_threshold[j] = true;
        start_threshold[j] = outc[j].rerun_threshold;
        rerun = true;
      }
    }
    if (rerun && trace) continue;  // a traced job is one job: run it again whole

    const uint64_t t_loop = now_ns();
    const uint64_t t_attempt = t_launch - t_setup;  // uploads (and tiles) of this attempt
    runs.assign(nj, Run{});
    std::vector<size_t> again;  // overflowed jobs of a batch run again alone, the rest finish now
    for (size_t j = 0; j < nj; ++j) {
      if (outc[j].rerun) {
        again.push_back(j);
        continue;
      }
      const unsigned long long* cj = &cnt[j * kNumCounters];
      const uint64_t n = std::min<uint64_t>(cj[kCandidates], capacity[j]);
      Run& r = runs[j];
      r.prec = pjs[j].prec;
      r.n_parts = pjs[j].desc.n_parts;
      r.parts = pjs[j].parts;
      r.tsz = pjs[j].tsz;
      Outcome& o = outc[j];
      r.levels_exact = o.levels_exact;
      r.candidates = cj[kCandidates];
      r.truncated = cj[kRecordsFull] != 0 || r.candidates > capacity[j];
      const Cand* d_cands = reinterpret_cast<const Cand*>(static_cast<const uint8_t*>(ws->records.p) + rec_off[j]);
      finish_selection(ws->select, ws->stream, pjs[j], descs[j], d_cands, n, recs[j], o, !cj[kLevelOverflow], r,
                       d2h_bytes);
      r.level_value = std::move(o.value);
      r.level_count = std::move(o.count);
      r.level_checksum = std::move(o.checksum);
      r.stats.finished = cj[kFinished];
      r.stats.working = 0;
      if (r.count) {
        r.stats.best_objective =
            pjs[j].prec == 1 ? read_t<double>(r.objective.data()) : static_cast<double>(read_t<float>(r.objective.data()));
        r.stats.best_rank = r.id[0];
      } else {
        r.stats.best_objective = std::numeric_limits<double>::infinity();
      }
    }
    for (size_t j = 0; j < nj; ++j) {
      runs[j].h2d_bytes = h2d_bytes / nj;
      runs[j].d2h_bytes = d2h_bytes / nj;
    }
    if (!again.empty()) {
      std::vector<PreparedJob> sub;
      std::vector<const sqsg_job*> subsrc;
      for (size_t j : again) {
        PreparedJob pj = pjs[j];
        pj.rerun_capacity = capacity[j];
        pj.rerun_slots = slots[j];
        pj.rerun_threshold = start_threshold[j];
        pj.passes += attempt + 1;
        sub.push_back(std::move(pj));
        subsrc.push_back(srcs[j]);
      }
      std::vector<Run> subruns;
      execute(sub, subsrc, device, subruns, nullptr);
      for (size_t k = 0; k < again.size(); ++k) {
        const uint64_t total = subruns[k].stats.timings_ns[SQSG_TIMING_LOOP];
        runs[again[k]] = std::move(subruns[k]);
        runs[again[k]].stats.timings_ns[SQSG_TIMING_LOOP] = total + static_cast<uint64_t>(loop_ms_total * 1e6);
      }
    }
    if (trace && trace->capacity) {
      const PreparedJob& pj = pjs[0];
      const uint64_t n = std::min<uint64_t>(pj.range_count, trace->capacity);
      if (trace->count) *trace->count = pj.range_count;
      const JobDesc& d = pj.desc;
      if (trace->species)
        CUDA_CHECK(cudaMemcpy(trace->species, ws->trace_sp.p, n * d.trace_species_stride, cudaMemcpyDeviceToHost));
      if (trace->bonds)
        CUDA_CHECK(cudaMemcpy(trace->bonds, ws->trace_bd.p, n * d.trace_bonds_stride * 4, cudaMemcpyDeviceToHost));
      if (trace->objective)
        CUDA_CHECK(cudaMemcpy(trace->objective, ws->trace_obj.p, n * pj.tsz, cudaMemcpyDeviceToHost));
      if (trace->id) CUDA_CHECK(cudaMemcpy(trace->id, ws->trace_id.p, n * 8, cudaMemcpyDeviceToHost));
    }
    const uint64_t t_end = now_ns();
    for (size_t j = 0; j < nj; ++j) {
      uint64_t* st = runs[j].stage_ns;
      if (st[SQSG_STAGE_TOTAL]) continue;  // a job that ran again alone keeps its own profile
      st[SQSG_STAGE_PREPARE] = pjs[j].prepare_ns + (t_setup - t0);
      st[SQSG_STAGE_UPLOAD] = t_attempt;
      st[SQSG_STAGE_KERNEL] = static_cast<uint64_t>(loop_ms_total * 1e6);
      st[SQSG_STAGE_WAIT] = t_done - t_launch;
      st[SQSG_STAGE_LEVELS] = t_loop - t_done;
      st[SQSG_STAGE_SELECT] = t_end - t_loop;
      st[SQSG_STAGE_TOTAL] = pjs[j].prepare_ns + (t_end - t0);
    }
    std::vector<bool> rerun_job(nj, false);
    for (size_t j : again) rerun_job[j] = true;
    for (size_t j = 0; j < nj; ++j) {
      Run& r = runs[j];
      r.stats.timings_ns[SQSG_TIMING_TOTAL] = t_end - t0;
      r.stats.timings_ns[SQSG_TIMING_CHUNK_SETUP] = t_setup - t0;
      if (!rerun_job[j]) r.stats.timings_ns[SQSG_TIMING_LOOP] = static_cast<uint64_t>(loop_ms_total * 1e6);
      r.stats.timings_ns[SQSG_TIMING_COMM] = t_end - t_loop;
    }
    return;
  }
}


// ------------------------------------------------------------------------------------------------
// Served form: continuous batching on a live tile ring.
//
// Jobs are submitted at any time. The server's worker thread admits a job when a job slot, ring
// space and device memory for its data and records are free (admission by footprint), uploads it
// on a copy stream, appends its tiles to the ring of its shared-memory bucket and raises the ring's
// tail; the bucket's persistent kernel, already running other jobs' tiles, picks them up. The CTA
// that finishes a job's last tile marks the job's slot done in host-mapped memory; the worker then
// downloads its records and levels, selects the result set and wakes the waiting caller. A job's
// result does not depend on what else runs: its tiles and random words depend only on the job.
// One ring per (kernel, occupancy level): ring 0 runs sqsg_engine_mask at 5 CTAs per SM and takes
// binary bit-mask jobs; rings 1-4 run sqsg_engine_wide at 4, 3, 2, 1 CTAs per SM; rings 5-6 run
// sqsg_engine_lat2 at 4 and 2, rings 7-8 sqsg_engine_lat5 at 3 and 1, rings 9-10 sqsg_engine_lat at 2
// and 1, rings 11-12 sqsg_engine_latw at 2 and 1 CTAs per SM. A job goes to the ring of its kernel
// with the largest shared-memory size it fits, i.e. the highest occupancy its data allow; a bit-mask
// job that fits no mask ring may take a wide ring, and a lattice job of up to 64 cells that fits no
// ring of its kernel a ring of sqsg_engine_lat.
constexpr int kBuckets = 13;
struct RingSpec {
  int kind;  // KernelKind
  int want;  // CTAs per SM
};
constexpr RingSpec kRingSpec[kBuckets] = {{kKindMask, 5}, {kKindWide, 4}, {kKindWide, 3}, {kKindWide, 2},
                                          {kKindWide, 1}, {kKindLat2, 4}, {kKindLat2, 2}, {kKindLat5, 3},
                                          {kKindLat5, 1}, {kKindLat, 2},  {kKindLat, 1},  {kKindLatW, 2},
                                          {kKindLatW, 1}};
// CTAs per SM of the most occupied ring of a kernel kind.
static int ring_top_occupancy(int kind) {
  int top = 1;
  for (const RingSpec& r : kRingSpec)
    if (r.kind == kind) top = std::max(top, r.want);
  return top;
}
constexpr int kMaxSm = 256;
constexpr size_t kOnesBytes = 1u << 20;  // pinned 0xff source of distinct-configuration table resets
constexpr uint64_t kRingCap = 1u << 20;
constexpr uint32_t kIdlePolls = 2500;         // ~5 ms of empty polls before a CTA leaves its ring
constexpr int kLaunchSlots = 32;              // concurrent launches per ring
constexpr uint64_t kRepartitionNs = 5000000;  // at most one SM repartition per 5 ms
constexpr uint64_t kRelaunchNs = 1000000;     // at most one top-up launch per ring per ms
constexpr uint8_t kNoOwner = 0xff;
constexpr int kReservedSm = 16;               // SMs left to no ring: result selection runs there
constexpr double kTilePairs = 1u << 19;       // estimated pair evaluations per thread and tile, at most

struct ServerJob {
  uint64_t ticket = 0;
  uint32_t slot = 0, gen = 0;
  int bucket = 0;
  PreparedJob pj;
  std::vector<Tile> tiles;
  std::vector<uint64_t> cum;  // cum[k] = configurations in tiles[0, k)
  double cost = 1.0;          // estimated cost of a configuration in pair evaluations (config_cost)
  size_t arena_off = 0, arena_bytes = 0, blob_bytes = 0;
  uint64_t capacity = 0;
  uint64_t slots = 0;         // > 0: deduplicating re-run (distinct-configuration table after the records)
  bool user_capacity = false;
  int attempt = 0;
  bool fixed_threshold = false;
  double start_threshold = 0.0;
  uint64_t ring_begin = 0, ring_end = 0;
  uint64_t t_submit = 0, t_admit = 0;
  uint64_t h2d_bytes = 0;
  JobDesc dev_desc{};         // the descriptor as uploaded (device pointers into the arena)
};

struct LaunchSlot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
};

// One ring of tiles per shared-memory class; launches of its kernel serve a ring on the SMs that
// the owner table gives it.
struct Ring {
  EngineKernel kernel = nullptr;  // ring 0: sqsg_engine_mask (bit-mask jobs); others: sqsg_engine_wide
  size_t smem = 0;
  uint32_t per_sm = 1;        // resident CTAs per SM at this shared-memory size
  uint64_t published = 0;     // tiles appended so far (the ring's tail)
  uint32_t launched = 0;      // CTAs launched so far (wraps like QueueCtl::exited)
  uint64_t last_launch = 0;
  LaunchSlot ls[kLaunchSlots];
};

struct ServerState {
  int device = 0;
  int n_sm = 0;
  sqsg_server_options opt{};
  cudaStream_t copy = nullptr;
  Ring rings[kBuckets];
  uint8_t* arena = nullptr;
  std::map<size_t, size_t> free_list;  // offset -> size
  JobDesc* d_jobs = nullptr;
  unsigned long long* d_counters = nullptr;
  LevelSlot* d_levels = nullptr;
  Tile* d_ring[kBuckets] = {};
  // d_ctl: kBuckets QueueCtl, the device status word (64 B), kBuckets x kMaxSm alive counters
  uint8_t* d_ctl = nullptr;
  uint8_t* h_ctl = nullptr;     // pinned mirror of d_ctl
  uint8_t* d_owner = nullptr;   // owner ring of each SM
  uint8_t* h_owner = nullptr;   // pinned: the table as last written
  uint64_t last_partition = 0;
  uint32_t* h_yield = nullptr;  // pinned sources of yield writes
  uint8_t* h_zero = nullptr;    // pinned zeros: level tables are cleared by copy, not by a kernel
  uint8_t* h_ones = nullptr;    // pinned 0xff bytes (kOnesBytes): empty distinct-configuration tables
  uint32_t* h_done = nullptr;
  uint32_t* d_done = nullptr;
  std::vector<std::unique_ptr<ServerJob>> slots;
  std::vector<uint32_t> slot_gen;
  std::deque<std::unique_ptr<ServerJob>> pending;
  std::map<uint64_t, Run> finished;
  std::map<uint64_t, std::pair<sqsg_status, std::string>> failed;
  std::string broken;  // set after a device error: the server fails every job from then on
  struct Collected {    // a finished job's counters and levels, downloaded; selected by a finalizer thread
    std::unique_ptr<ServerJob> job;
    std::vector<unsigned long long> cnt;
    std::vector<LevelSlot> levels;
    std::vector<Cand> records;
  };
  std::deque<Collected> collected;
  std::mutex m;
  std::condition_variable cv_work, cv_done, cv_fin;
  std::thread worker;
  std::vector<std::thread> finalizers;
  bool stop = false;
  uint64_t next_ticket = 1;
  sqsg_server_counters stats{};
  QueueCtl* q(int b) const { return reinterpret_cast<QueueCtl*>(d_ctl) + b; }
  const QueueCtl& hq(int b) const { return reinterpret_cast<const QueueCtl*>(h_ctl)[b]; }
  unsigned long long device_status() const {
    return *reinterpret_cast<const unsigned long long*>(h_ctl + kBuckets * sizeof(QueueCtl));
  }
  unsigned int* d_alive(int b) const {
    return reinterpret_cast<unsigned int*>(d_ctl + kBuckets * sizeof(QueueCtl) + 64) + static_cast<size_t>(b) * kMaxSm;
  }
  const unsigned int* h_alive(int b) const {
    return reinterpret_cast<const unsigned int*>(h_ctl + kBuckets * sizeof(QueueCtl) + 64) +
           static_cast<size_t>(b) * kMaxSm;
  }
};

constexpr size_t kCtlBytes = kBuckets * sizeof(QueueCtl) + 64 + kBuckets * kMaxSm * sizeof(unsigned int);

static bool arena_alloc(ServerState& S, size_t bytes, size_t* off) {
  bytes = align_up(bytes, 256);
  for (auto it = S.free_list.begin(); it != S.free_list.end(); ++it) {
    if (it->second >= bytes) {
      *off = it->first;
      const size_t rest = it->second - bytes;
      const size_t roff = it->first + bytes;
      S.free_list.erase(it);
      if (rest) S.free_list[roff] = rest;
      return true;
    }
  }
  return false;
}

static void arena_free(ServerState& S, size_t off, size_t bytes) {
  bytes = align_up(bytes, 256);
  auto it = S.free_list.emplace(off, bytes).first;
  auto next = std::next(it);
  if (next != S.free_list.end() && it->first + it->second == next->first) {
    it->second += next->second;
    S.free_list.erase(next);
  }
  if (it != S.free_list.begin()) {
    auto prev = std::prev(it);
    if (prev->first + prev->second == it->first) {
      prev->second += it->second;
      S.free_list.erase(it);
    }
  }
}

static size_t job_footprint(const ServerJob& J) {
  return align_up(J.pj.blob.size(), 256) + align_up(J.capacity * sizeof(Cand), 256) +
         align_up(J.slots * sizeof(DedupSlot), 256);
}

// Admits the oldest pending job if a slot, ring space and arena memory are free: uploads its data,
// counters, level table, descriptor and tiles on the copy stream, then raises its ring's tail.
// Called with S.m held.
static bool try_admit(ServerState& S) {
  if (S.pending.empty()) return false;
  ServerJob& J = *S.pending.front();
  uint32_t slot = static_cast<uint32_t>(S.slots.size());
  for (uint32_t k = 0; k < S.slots.size(); ++k)
    if (!S.slots[k]) {
      slot = k;
      break;
    }
  if (slot == S.slots.size()) return false;
  const int b = J.bucket;
  Ring& R = S.rings[b];
  uint64_t oldest = R.published;  // ring entries before the oldest live job's tiles are free
  for (auto& x : S.slots)
    if (x && x->bucket == b) oldest = std::min(oldest, x->ring_begin);
  if (R.published + J.tiles.size() - oldest > kRingCap) return false;
  J.blob_bytes = align_up(J.pj.blob.size(), 256);
  J.arena_bytes = job_footprint(J);
  if (!arena_alloc(S, J.arena_bytes, &J.arena_off)) return false;
  J.slot = slot;
  J.gen = ++S.slot_gen[slot];
  if (J.gen == 0) J.gen = ++S.slot_gen[slot];
  J.t_admit = now_ns();
  JobDesc d = J.pj.desc;
  d.blob = S.arena + J.arena_off;
  d.records = S.arena + J.arena_off + J.blob_bytes;
  d.capacity = J.capacity;
  d.counters = S.d_counters + static_cast<size_t>(slot) * kNumCounters;
  d.levels = S.d_levels + static_cast<size_t>(slot) * kLevelSlots;
  std::vector<unsigned long long> init(kNumCounters, 0);
  const double maxv = J.pj.prec == 1 ? std::numeric_limits<double>::max()
                                     : static_cast<double>(std::numeric_limits<float>::max());
  init[kThreshold] = ord_bits(J.fixed_threshold ? J.start_threshold : maxv);
  init[kBest] = ord_bits(std::numeric_limits<double>::infinity());
  init[kTilesLeft] = J.tiles.size();
  for (auto& t : J.tiles) {
    t.job = slot;
    t.gen = J.gen;
  }
  CUDA_CHECK(cudaMemcpyAsync(S.arena + J.arena_off, J.pj.blob.data(), J.pj.blob.size(), cudaMemcpyHostToDevice, S.copy));
  CUDA_CHECK(cudaMemcpyAsync(d.counters, init.data(), init.size() * 8, cudaMemcpyHostToDevice, S.copy));
  // copies only: a memset kernel would wait for SMs held by the running persistent kernels
  CUDA_CHECK(cudaMemcpyAsync(d.levels, S.h_zero, kLevelSlots * sizeof(LevelSlot), cudaMemcpyHostToDevice, S.copy));
  if (J.slots) {  // the distinct-configuration table starts empty (all bits set), also by copies
    d.dedup = reinterpret_cast<DedupSlot*>(d.records + align_up(J.capacity * sizeof(Cand), 256));
    d.dedup_mask = J.slots - 1;
    const size_t bytes = J.slots * sizeof(DedupSlot);
    for (size_t off = 0; off < bytes; off += kOnesBytes)
      CUDA_CHECK(cudaMemcpyAsync(reinterpret_cast<uint8_t*>(d.dedup) + off, S.h_ones,
                                 std::min<size_t>(kOnesBytes, bytes - off), cudaMemcpyHostToDevice, S.copy));
  }
  CUDA_CHECK(cudaMemcpyAsync(S.d_jobs + slot, &d, sizeof(d), cudaMemcpyHostToDevice, S.copy));
  J.dev_desc = d;
  const uint64_t n = J.tiles.size();
  const uint64_t pos = R.published % kRingCap;
  const uint64_t first = std::min<uint64_t>(n, kRingCap - pos);
  if (first)
    CUDA_CHECK(cudaMemcpyAsync(S.d_ring[b] + pos, J.tiles.data(), first * sizeof(Tile), cudaMemcpyHostToDevice, S.copy));
  if (n > first)
    CUDA_CHECK(cudaMemcpyAsync(S.d_ring[b], J.tiles.data() + first, (n - first) * sizeof(Tile), cudaMemcpyHostToDevice,
                               S.copy));
  J.ring_begin = R.published;
  R.published += n;
  J.ring_end = R.published;
  // the tail rises only after everything above is in device memory (same stream)
  const unsigned long long tail = R.published;
  CUDA_CHECK(cudaMemcpyAsync(&S.q(b)->tail, &tail, sizeof(tail), cudaMemcpyHostToDevice, S.copy));
  CUDA_CHECK(cudaStreamSynchronize(S.copy));
  J.h2d_bytes += J.pj.blob.size() + init.size() * 8 + sizeof(d) + n * sizeof(Tile) + sizeof(tail);
  S.slots[slot] = std::move(S.pending.front());
  S.pending.pop_front();
  S.stats.admitted++;
  return true;
}

// Candidate records a (re-)run of J may keep in the arena: the re-run budget, and what the arena holds
// next to the job's own data.
static uint64_t arena_record_limit(const ServerState& S, const ServerJob& J) {
  const uint64_t arena_bytes = S.opt.arena_bytes;
  return std::min<uint64_t>(rerun_limit(J.pj),
                            (arena_bytes - std::min<uint64_t>(arena_bytes, align_up(J.pj.blob.size(), 256) + 256)) /
                                sizeof(Cand));
}

// Puts a job whose candidate buffer overflowed back at the front of the queue, with the threshold,
// buffer and distinct-configuration table that assess() asks for (the same configurations are
// evaluated again). Called with S.m held, after the job's arena memory was released.
static void requeue_rerun(ServerState& S, std::unique_ptr<ServerJob> job, const Outcome& o) {
  ServerJob& J = *job;
  J.capacity = o.rerun_capacity;
  J.slots = o.rerun_slots;
  J.fixed_threshold = true;
  J.start_threshold = o.rerun_threshold;
  J.attempt++;
  S.pending.push_front(std::move(job));
  S.cv_work.notify_one();
}

// Collects a finished job on the worker thread: counters and level table come back on the copy
// stream (the records too when the level table overflowed) and the job's slot is released at once.
// A job that must run again with an exact level table is requeued here (the decision reads only the
// counters and the level table), not behind the finalizers, which may be busy with large result
// sets. Otherwise its arena memory stays with it until a finalizer thread has selected the result
// set, so that admission and launches go on meanwhile.
static void collect(ServerState& S, uint32_t slot) {
  ServerState::Collected c;
  c.job = std::move(S.slots[slot]);
  ServerJob& J = *c.job;
  c.cnt.resize(kNumCounters);
  CUDA_CHECK(cudaMemcpyAsync(c.cnt.data(), S.d_counters + static_cast<size_t>(slot) * kNumCounters,
                             c.cnt.size() * 8, cudaMemcpyDeviceToHost, S.copy));
  c.levels.resize(kLevelSlots);
  CUDA_CHECK(cudaMemcpyAsync(c.levels.data(), S.d_levels + static_cast<size_t>(slot) * kLevelSlots,
                             kLevelSlots * sizeof(LevelSlot), cudaMemcpyDeviceToHost, S.copy));
  CUDA_CHECK(cudaStreamSynchronize(S.copy));
  const uint64_t n = std::min<uint64_t>(c.cnt[kCandidates], J.capacity);
  if (c.cnt[kLevelOverflow] && n) {
    c.records.resize(n);
    CUDA_CHECK(cudaMemcpyAsync(c.records.data(), S.arena + J.arena_off + J.blob_bytes, n * sizeof(Cand),
                               cudaMemcpyDeviceToHost, S.copy));
    CUDA_CHECK(cudaStreamSynchronize(S.copy));
  }
  if (!J.slots && !c.cnt[kLevelOverflow]) {
    Outcome o;
    bool decided = false;
    try {
      check_job_counters(c.cnt.data());
      o = assess(J.pj, c.cnt.data(), c.levels.data(), c.records, n, J.capacity, !J.user_capacity && J.attempt < 2,
                 arena_record_limit(S, J));
      decided = true;
    } catch (std::exception const&) {
      // the finalizer reports the job's error
    }
    if (decided && o.rerun) {
      arena_free(S, J.arena_off, J.arena_bytes);
      requeue_rerun(S, std::move(c.job), o);
      return;
    }
  }
  S.collected.push_back(std::move(c));
  S.cv_fin.notify_one();
}

// Finalizer thread: selects a collected job's result set like sqsg_optimize selects it (on the
// device from the job's arena records, on its own stream, for large sets), or, when its record
// buffer overflowed, puts it back at the front of the queue with the threshold and buffer that
// assess() asks for (the same configurations are evaluated again).
static void finalizer_loop(ServerState* Sp) {
  ServerState& S = *Sp;
  cudaSetDevice(S.device);
  cudaStream_t stream = nullptr;
  SelectScratch scratch;
  std::unique_lock<std::mutex> lock(S.m);
  if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    stream = nullptr;
    if (S.broken.empty()) S.broken = "a finalizer could not create its stream";
  }
  while (true) {
    S.cv_fin.wait(lock, [&] { return S.stop || !S.collected.empty(); });
    if (S.stop) break;
    ServerState::Collected c = std::move(S.collected.front());
    S.collected.pop_front();
    lock.unlock();
    ServerJob& J = *c.job;
    std::string error;
    if (J.slots && stream) {  // a deduplicating re-run: its distinct configurations are the candidates
      try {
        c.cnt[kCandidates] = compact_dedup(scratch, stream, J.dev_desc.dedup, J.slots,
                                           reinterpret_cast<Cand*>(S.arena + J.arena_off + J.blob_bytes), J.capacity);
      } catch (std::exception const& ex) {
        error = ex.what();
      }
    }
    const unsigned long long* cnt = c.cnt.data();
    const uint64_t n = std::min<uint64_t>(cnt[kCandidates], J.capacity);
    const uint64_t arena_records = arena_record_limit(S, J);
    Run r;
    Outcome o;
    uint64_t fin_d2h = c.records.size() * sizeof(Cand);
    try {
      if (!error.empty()) throw cuda_error(error);
      check_job_counters(cnt);
      o = assess(J.pj, cnt, c.levels.data(), c.records, n, J.capacity, !J.user_capacity && J.attempt < 2,
                 arena_records);
      if (!o.rerun) {
        r.prec = J.pj.prec;
        r.n_parts = J.pj.desc.n_parts;
        r.parts = J.pj.parts;
        r.tsz = J.pj.tsz;
        r.levels_exact = o.levels_exact;
        r.candidates = cnt[kCandidates];
        r.truncated = cnt[kRecordsFull] != 0 || r.candidates > J.capacity;
        if (!stream) throw cuda_error("no stream to select the result set on");
        const Cand* d_cands = reinterpret_cast<const Cand*>(S.arena + J.arena_off + J.blob_bytes);
        finish_selection(scratch, stream, J.pj, J.dev_desc, d_cands, n, c.records, o, !cnt[kLevelOverflow], r,
                         fin_d2h);
        r.level_value = std::move(o.value);
        r.level_count = std::move(o.count);
        r.level_checksum = std::move(o.checksum);
        r.stats.finished = cnt[kFinished];
        if (r.count) {
          r.stats.best_objective = J.pj.prec == 1 ? read_t<double>(r.objective.data())
                                                  : static_cast<double>(read_t<float>(r.objective.data()));
          r.stats.best_rank = r.id[0];
        } else {
          r.stats.best_objective = std::numeric_limits<double>::infinity();
        }
        const uint64_t t_end = now_ns();
        r.stats.timings_ns[SQSG_TIMING_TOTAL] = t_end - J.t_submit;  // latency: submission to result
        r.stats.timings_ns[SQSG_TIMING_CHUNK_SETUP] = J.t_admit - J.t_submit;
        r.stats.timings_ns[SQSG_TIMING_LOOP] = t_end - J.t_admit;
        r.h2d_bytes = J.h2d_bytes;
        r.d2h_bytes = kLevelSlots * sizeof(LevelSlot) + kNumCounters * 8 + fin_d2h;
      }
    } catch (std::exception const& ex) {
      error = ex.what();
    }
    lock.lock();
    arena_free(S, J.arena_off, J.arena_bytes);
    if (!error.empty()) {
      S.failed[J.ticket] = {SQSG_ERR_CUDA, error};
      S.cv_done.notify_all();
    } else if (o.rerun) {
      requeue_rerun(S, std::move(c.job), o);
    } else {
      S.stats.completed++;
      S.stats.configurations += cnt[kFinished];
      S.finished.emplace(J.ticket, std::move(r));
      S.cv_done.notify_all();
    }
  }
  lock.unlock();
  scratch.release();
  if (stream) {
    cudaStreamSynchronize(stream);
    cudaStreamDestroy(stream);
  }
}

// Partitions the SMs (all but kReservedSm) between the rings that hold unclaimed tiles, in
// proportion to their outstanding work in SM-time (pair evaluations of the unclaimed tiles over the
// ring's CTAs per SM), so that every SM runs CTAs of one shared-memory size at that size's full
// occupancy. A ring whose SMs hold fewer of its CTAs than they can take gets a launch of a full
// grid; CTAs that land on another ring's SM leave at once, and CTAs leave between tiles when their
// SM changes hands.
static void schedule(ServerState& S) {
  const uint64_t now = now_ns();
  double work[kBuckets] = {};
  double total = 0.0;
  int n_want = 0;
  for (auto& x : S.slots) {
    if (!x) continue;
    const uint64_t head = S.hq(x->bucket).head;
    if (head >= x->ring_end) continue;
    const uint64_t k0 = head > x->ring_begin ? head - x->ring_begin : 0;
    const double configs = static_cast<double>(x->cum.back() - x->cum[k0]);
    // SM-time: the cost is measured at the kernel's highest occupancy; a ring of fewer CTAs per SM
    // takes proportionally longer per configuration
    work[x->bucket] += configs * x->cost * ring_top_occupancy(kRingSpec[x->bucket].kind) / S.rings[x->bucket].per_sm;
  }
  for (int b = 0; b < kBuckets; ++b) {
    total += work[b];
    n_want += work[b] > 0 ? 1 : 0;
  }
  if (!n_want) return;
  const int n_sm = S.n_sm - kReservedSm;
  int cur[kBuckets] = {};
  for (int sm = 0; sm < n_sm; ++sm)
    if (S.h_owner[sm] < kBuckets) cur[S.h_owner[sm]]++;
  int want[kBuckets] = {};
  double frac[kBuckets] = {};
  int given = 0;
  for (int b = 0; b < kBuckets; ++b) {
    if (work[b] <= 0) continue;
    const double share = n_sm * work[b] / total;
    want[b] = std::max(1, static_cast<int>(share));
    frac[b] = share - static_cast<int>(share);
    given += want[b];
  }
  while (given < n_sm) {  // hand out the remainder by largest fractional share
    int best = -1;
    for (int b = 0; b < kBuckets; ++b)
      if (work[b] > 0 && (best < 0 || frac[b] > frac[best])) best = b;
    want[best]++;
    frac[best] -= 1.0;
    given++;
  }
  while (given > n_sm) {  // rings held at one SM each took too many: trim the largest
    int big = 0;
    for (int b = 1; b < kBuckets; ++b)
      if (want[b] > want[big]) big = b;
    want[big]--;
    given--;
  }
  bool change = false;
  for (int b = 0; b < kBuckets; ++b) {
    if (work[b] > 0 && cur[b] == 0) change = true;
    if (work[b] <= 0 && cur[b] > 0) change = true;
    if (std::abs(want[b] - cur[b]) > std::max(2, cur[b] / 4)) change = true;
  }
  if (change && now - S.last_partition > kRepartitionNs) {
    std::vector<int> pool;  // SMs to hand out: unowned, of rings without work, or a ring's excess
    for (int sm = n_sm - 1; sm >= 0; --sm) {
      const uint8_t o = S.h_owner[sm];
      if (o >= kBuckets || work[o] <= 0 || cur[o] > want[o]) {
        if (o < kBuckets && work[o] > 0) cur[o]--;
        S.h_owner[sm] = kNoOwner;
        pool.push_back(sm);
      }
    }
    for (int b = 0; b < kBuckets; ++b) cur[b] = 0;
    for (int sm = 0; sm < n_sm; ++sm)
      if (S.h_owner[sm] < kBuckets) cur[S.h_owner[sm]]++;
    for (int b = 0; b < kBuckets; ++b)
      while (cur[b] < want[b] && !pool.empty()) {
        S.h_owner[pool.back()] = static_cast<uint8_t>(b);
        pool.pop_back();
        cur[b]++;
      }
    CUDA_CHECK(cudaMemcpyAsync(S.d_owner, S.h_owner, kMaxSm, cudaMemcpyHostToDevice, S.copy));
    CUDA_CHECK(cudaStreamSynchronize(S.copy));
    S.last_partition = now;
  }
  for (int b = 0; b < kBuckets; ++b) {
    if (work[b] <= 0) continue;
    Ring& R = S.rings[b];
    uint64_t room = 0;
    const unsigned int* alive = S.h_alive(b);
    for (int sm = 0; sm < n_sm; ++sm)
      if (S.h_owner[sm] == b && alive[sm] < R.per_sm) room += R.per_sm - alive[sm];
    if (room < R.per_sm || now - R.last_launch < kRelaunchNs) continue;  // top up by whole SMs
    for (auto& L : R.ls) {
      if (L.busy) continue;
      const uint32_t grid = R.per_sm * static_cast<uint32_t>(S.n_sm);
      R.kernel<<<grid, kBlock, R.smem, L.stream>>>(
          S.d_jobs, S.d_ring[b], 0, S.q(b), nullptr,
          reinterpret_cast<unsigned long long*>(S.d_ctl + kBuckets * sizeof(QueueCtl)), S.d_done);
      CUDA_CHECK(cudaGetLastError());
      CUDA_CHECK(cudaEventRecord(L.done, L.stream));
      L.busy = true;
      R.launched += grid;
      R.last_launch = now;
      S.stats.launches++;
      break;
    }
  }
}

static void fail_all(ServerState& S, const std::string& why) {
  for (auto& x : S.slots)
    if (x) {
      S.failed[x->ticket] = {SQSG_ERR_CUDA, why};
      x.reset();
    }
  while (!S.pending.empty()) {
    S.failed[S.pending.front()->ticket] = {SQSG_ERR_CUDA, why};
    S.pending.pop_front();
  }
  S.cv_done.notify_all();
}

static void server_loop(ServerState* Sp) {
  ServerState& S = *Sp;
  cudaSetDevice(S.device);
  std::unique_lock<std::mutex> lock(S.m);
  while (!S.stop) {
    bool progress = false;
    if (S.broken.empty()) {
      try {
        // the control block comes back without the lock held: only this thread uses the copy stream
        // and changes the slots it describes, and submissions and finalizers need not wait for a copy
        // engine that may be busy with large result sets
        lock.unlock();
        cudaError_t ce = cudaMemcpyAsync(S.h_ctl, S.d_ctl, kCtlBytes, cudaMemcpyDeviceToHost, S.copy);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(S.copy);
        lock.lock();
        CUDA_CHECK(ce);
        if (const unsigned long long st = S.device_status())
          throw cuda_error("device error " + std::to_string(st) + " in the serving kernel");
        for (uint32_t k = 0; k < S.slots.size(); ++k) {
          if (!S.slots[k]) continue;
          if (*reinterpret_cast<volatile uint32_t*>(&S.h_done[k]) == S.slots[k]->gen) {
            collect(S, k);
            progress = true;
          }
        }
        while (try_admit(S)) progress = true;
        for (auto& R : S.rings)
          for (auto& L : R.ls) {
            if (!L.busy) continue;
            const cudaError_t e = cudaEventQuery(L.done);
            if (e == cudaErrorNotReady) continue;
            CUDA_CHECK(e);
            L.busy = false;
            progress = true;
          }
        schedule(S);
      } catch (std::exception const& ex) {
        // A device error leaves CTAs of failed jobs possibly still running over arena memory that
        // must not be handed out again: the server stops serving and fails every job.
        S.broken = ex.what();
        fail_all(S, S.broken);
      }
    } else if (!S.pending.empty()) {
      fail_all(S, S.broken);
    }
    if (!progress) S.cv_work.wait_for(lock, std::chrono::microseconds(50));
  }
}

}  // namespace sqsg

using namespace sqsg;

struct sqsg_run {
  Run r;
};

extern "C" {

const char* sqsg_version(void) { return "sqsgen_b200 0.2.0 (abi 2, sm_100a)"; }

size_t sqsg_last_error(char* buf, size_t len) {
  const std::string& e = g_last_error;
  if (buf && len) {
    size_t n = std::min(len - 1, e.size());
    std::memcpy(buf, e.data(), n);
    buf[n] = 0;
  }
  return e.size();
}

int sqsg_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

sqsg_status sqsg_num_permutations(const uint8_t* conf, uint32_t n, uint64_t* out) {
  return guarded([&] {
    if ((!conf && n) || !out) throw std::invalid_argument("null pointer");
    uint32_t counts[256] = {0};
    for (uint32_t i = 0; i < n; ++i) counts[conf[i]]++;
    std::vector<uint32_t> dense;
    for (uint32_t v = 0; v < 256; ++v)
      if (counts[v]) dense.push_back(counts[v]);
    if (!num_permutations_counts(dense.data(), static_cast<int>(dense.size()), out))
      throw std::out_of_range("The number of permutations does not fit in 64 bits");
  });
}

sqsg_status sqsg_rank_permutation(const uint8_t* conf, uint32_t n, uint64_t* rank) {
  return guarded([&] {
    if ((!conf && n) || !rank) throw std::invalid_argument("null pointer");
    int k = 0;
    for (uint32_t i = 0; i < n; ++i) k = std::max(k, conf[i] + 1);
    uint64_t total;
    sqsg_status s = sqsg_num_permutations(conf, n, &total);
    if (s != SQSG_OK) throw std::out_of_range("The number of permutations does not fit in 64 bits");
    std::vector<uint32_t> hist(std::max(k, 1));
    *rank = rank_permutation(conf, n, hist.data(), k);
  });
}

sqsg_status sqsg_unrank_permutation(uint8_t* conf, uint32_t n, uint64_t rank) {
  return guarded([&] {
    if (!conf && n) throw std::invalid_argument("null pointer");
    uint32_t counts[256] = {0};
    for (uint32_t i = 0; i < n; ++i) counts[conf[i]]++;
    std::vector<uint32_t> h;
    for (uint32_t v = 0; v < 256; ++v)
      if (counts[v]) h.push_back(counts[v]);
    uint64_t total;
    if (!num_permutations_counts(h.data(), static_cast<int>(h.size()), &total))
      throw std::out_of_range("The number of permutations does not fit in 64 bits");
    if (rank > total) throw std::out_of_range("The rank is larger than the total number of permutations");
    uint32_t pos = 0;
    for (uint32_t i = 0; i < n; i++)
      for (uint32_t j = 0; j < h.size(); j++) {
        uint64_t suffix = div_96x32(mul_64x32(total, h[j]), n - i, nullptr);
        if (rank <= suffix) {
          conf[pos++] = static_cast<uint8_t>(j);
          total = suffix;
          h[j]--;
          break;
        }
        rank -= suffix;
      }
  });
}

static sqsg_status run_jobs(const sqsg_job* jobs, uint32_t n, sqsg_run** out, const TraceOut* trace) {
  return guarded([&] {
    if (!jobs || !out || n == 0) throw std::invalid_argument("null pointer");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      throw cuda_error("no CUDA device is available (the optimiser has no CPU path)");
    }
    const int device = jobs[0].device;
    if (device < 0 || device >= ndev) throw std::invalid_argument("invalid device ordinal");
    std::vector<PreparedJob> pjs;
    std::vector<const sqsg_job*> srcs;
    for (uint32_t j = 0; j < n; ++j) {
      if (jobs[j].device != device) throw std::invalid_argument("a batch runs on one device");
      const uint64_t tp = now_ns();
      pjs.push_back(prepare(jobs[j], trace ? trace->capacity : 0));
      pjs.back().prepare_ns = now_ns() - tp;
      srcs.push_back(&jobs[j]);
    }
    if (n == 1 || trace) {
      std::vector<Run> runs;
      execute(pjs, srcs, device, runs, trace);
      for (uint32_t j = 0; j < n; ++j) out[j] = new sqsg_run{std::move(runs[j])};
      return;
    }
    // A batch runs as one persistent launch per occupancy class (kernel, CTAs per SM): a launch
    // takes the largest shared-memory size of its jobs, so mixing small and large jobs in one launch
    // would run the small ones at the large ones' occupancy.
    CUDA_CHECK(cudaSetDevice(device));
    configure_kernel(max_dynamic_smem(device));
    std::map<std::pair<int, int>, std::vector<uint32_t>> classes;
    for (uint32_t j = 0; j < n; ++j) {
      const int kind = kind_of(pjs[j].desc);
      int per_sm = 0;
      CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel_of(kind), kBlock,
                                                               pjs[j].desc.smem_bytes));
      classes[{kind, -per_sm}].push_back(j);
    }
    std::vector<std::unique_ptr<sqsg_run>> done(n);
    auto run_class = [&](const std::vector<uint32_t>& idx) {
      std::vector<PreparedJob> g;
      std::vector<const sqsg_job*> gs;
      for (uint32_t j : idx) {
        g.push_back(std::move(pjs[j]));
        gs.push_back(srcs[j]);
      }
      std::vector<Run> runs;
      execute(g, gs, device, runs, nullptr);
      for (size_t k = 0; k < idx.size(); ++k) done[idx[k]].reset(new sqsg_run{std::move(runs[k])});
    };
    // Classes run from one host thread each, on their own workspaces and streams: a class's persistent
    // kernel takes the SMs as the previous one's CTAs run out of tiles, and each class's result
    // selection overlaps the others' kernels. Progress callbacks are promised on the calling thread,
    // so a batch with any callback runs its classes one after another here.
    bool callbacks = false;
    for (uint32_t j = 0; j < n; ++j) callbacks |= jobs[j].callback != nullptr;
    if (callbacks || classes.size() == 1) {
      for (auto& [key, idx] : classes) run_class(idx);
    } else {
      std::vector<std::thread> threads;
      std::vector<std::exception_ptr> errors(classes.size());
      size_t k = 0;
      for (auto& [key, idx] : classes) {
        const std::vector<uint32_t>* ids = &idx;
        std::exception_ptr* err = &errors[k++];
        threads.emplace_back([&, ids, err] {
          try {
            CUDA_CHECK(cudaSetDevice(device));
            run_class(*ids);
          } catch (...) {
            *err = std::current_exception();
          }
        });
      }
      for (auto& t : threads) t.join();
      for (auto& e : errors)
        if (e) std::rethrow_exception(e);
    }
    for (uint32_t j = 0; j < n; ++j) out[j] = done[j].release();
  });
}

sqsg_status sqsg_set_option(const char* name, int64_t value) {
  return guarded([&] {
    const int k = option_index(name);
    if (k < 0) throw std::invalid_argument(std::string("unknown option: ") + (name ? name : "(null)"));
    if ((k == kOptStageWaitNs || k == kOptDefaultCandidates || k == kOptRerunRecordBytes ||
         k == kOptServerFinalizers) && value <= 0)
      throw std::out_of_range(std::string(kOptionNames[k]) + " must be positive");
    g_options[k].store(value);
  });
}

sqsg_status sqsg_get_option(const char* name, int64_t* value) {
  return guarded([&] {
    const int k = option_index(name);
    if (k < 0) throw std::invalid_argument(std::string("unknown option: ") + (name ? name : "(null)"));
    if (!value) throw std::invalid_argument("null pointer");
    *value = g_options[k].load();
  });
}

sqsg_status sqsg_plan_job(const sqsg_job* job, sqsg_plan* plan) {
  return guarded([&] {
    if (!job || !plan) throw std::invalid_argument("null pointer");
    PreparedJob pj = prepare(*job, 0);
    std::memset(plan, 0, sizeof(*plan));
    const JobDesc& d = pj.desc;
    plan->n_parts = d.n_parts;
    plan->smem_bytes = d.smem_bytes;
    plan->record_bytes = d.record_bytes;
    plan->bucket = bucket_key(*job);
    Tuning t;
    plan->tuned = option(kOptUseTuning) && tuning_lookup(plan->bucket, t) ? 1 : 0;
    const bool bitmask = d.k2 != 0;
    const int kind = kind_of(d);
    std::snprintf(plan->kernel, sizeof(plan->kernel), "%s", kernel_name(kind));
    for (uint32_t p = 0; p < d.n_parts; ++p) {
      const PartDesc& P = d.parts[p];
      plan->parts[p].path = bitmask ? SQSG_PATH_BITMASK : (d.lat ? SQSG_PATH_LATTICE : SQSG_PATH_GENERAL);
      plan->parts[p].stream_narrow = static_cast<int32_t>(P.stream_narrow);
      plan->parts[p].stream_staged = P.stream_global ? 0 : 1;
      if (d.lat) plan->parts[p].lattice_units = static_cast<uint32_t>(lattice_units(pj, p));
      if (!pj.systematic) {  // random words per configuration: Floyd windows draw m, the others n - 1
        const uint8_t* base = pj.blob.data() + P.blob_off + P.win_off;
        for (uint32_t w = 0; w < P.n_windows; ++w) {
          uint32_t lo, hi, fw;
          std::memcpy(&lo, base + 8ull * w, 4);
          std::memcpy(&hi, base + 8ull * w + 4, 4);
          std::memcpy(&fw, base + 8ull * P.n_windows + 4ull * w, 4);
          plan->shuffle_draws += fw ? (fw & 0xffffu) : hi - lo - 1;
        }
      }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) == cudaSuccess && job->device >= 0 && job->device < ndev) {
      CUDA_CHECK(cudaSetDevice(job->device));
      if (d.smem_bytes <= max_dynamic_smem(job->device)) {
        configure_kernel(d.smem_bytes);
        int per_sm = 0;
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel_of(kind), kBlock, d.smem_bytes));
        plan->ctas_per_sm = static_cast<uint32_t>(per_sm);
      }
    } else {
      cudaGetLastError();
    }
  });
}

sqsg_status sqsg_autotune(const sqsg_job* job, double seconds, sqsg_tuning* best, sqsg_tuning* tried,
                          uint32_t* n_tried) {
  return guarded([&] {
    if (!job || !best) throw std::invalid_argument("null pointer");
    if (!(seconds > 0)) throw std::out_of_range("seconds must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      throw cuda_error("no CUDA device is available (the autotuner measures on the device)");
    }
    const int device = job->device;
    if (device < 0 || device >= ndev) throw std::invalid_argument("invalid device ordinal");
    CUDA_CHECK(cudaSetDevice(device));
    sqsg_job probe = *job;
    probe.callback = nullptr;
    probe.cancel = nullptr;
    probe.max_results = 4096;  // the records are not what is timed
    const Tuning rules{};
    const PreparedJob base = prepare(probe, 0, &rules);
    const uint64_t total = base.range_count;
    if (total == 0) throw std::out_of_range("the job has no configurations to time");
    // the choices that apply to this job
    std::vector<std::pair<int, int>> paths;  // (path, stage)
    if (base.desc.lat) paths.push_back({SQSG_PATH_LATTICE, -1});
    if (base.desc.k2) paths.push_back({SQSG_PATH_BITMASK, -1});
    if (!base.desc.k2 && job->n_sublattices == 1) {
      paths.push_back({SQSG_PATH_GENERAL, 0});
      paths.push_back({SQSG_PATH_GENERAL, 1});
    } else if (!base.desc.k2) {
      paths.push_back({SQSG_PATH_GENERAL, 0});
    }
    std::vector<Tuning> cands;
    std::vector<int> cand_path;
    for (auto [path, stage] : paths) {
      Tuning t;
      t.path = path == SQSG_PATH_GENERAL ? SQSG_PATH_GENERAL : -1;
      t.stage = stage;
      const PreparedJob pj = prepare(probe, 0, &t);
      int per_sm = 0;
      configure_kernel(pj.desc.smem_bytes);
      CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel_of(kind_of(pj.desc)), kBlock,
                                                               pj.desc.smem_bytes));
      if (per_sm <= 0) continue;
      std::vector<uint32_t> ctas{0u};
      if (per_sm > 1) ctas.push_back(static_cast<uint32_t>(per_sm - 1));
      for (uint32_t c : ctas)
        for (uint32_t cap : {1024u, 8192u, 65536u}) {
          Tuning x = t;
          x.ctas = c;
          x.tile_cap = cap;
          cands.push_back(x);
          cand_path.push_back(path);
        }
    }
    auto timed = [&](const Tuning& t, uint64_t count) {
      probe.range_first = job->range_first;
      probe.range_count = count;
      std::vector<PreparedJob> pjs;
      pjs.push_back(prepare(probe, 0, &t));
      std::vector<const sqsg_job*> srcs{&probe};
      std::vector<Run> runs;
      execute(pjs, srcs, device, runs, nullptr);
      const double s = static_cast<double>(runs[0].stats.timings_ns[SQSG_TIMING_LOOP]) * 1e-9;
      return s > 0 ? static_cast<double>(runs[0].stats.finished) / s : 0.0;
    };
    // calibration with the rules (the first run also warms up), then equal shares of the budget
    const uint64_t c0 = std::min<uint64_t>(total, 1u << 22);
    timed(rules, c0);
    const double r0 = std::max(1.0, timed(rules, c0));
    const double share = seconds / (2.0 * std::max<size_t>(1, cands.size()));
    const uint64_t count = std::min<uint64_t>(total, std::max<uint64_t>(1u << 16, static_cast<uint64_t>(r0 * share)));
    std::vector<double> rate(cands.size());
    size_t bi = 0;
    for (size_t k = 0; k < cands.size(); ++k) {
      rate[k] = std::max(timed(cands[k], count), timed(cands[k], count));
      if (rate[k] > rate[bi]) bi = k;
    }
    if (cands.empty()) throw unsupported_error("no launch choice fits this job on the device");
    tuning_store(bucket_key(*job), cands[bi]);
    auto fill = [&](size_t k, sqsg_tuning& o) {
      o.path = cand_path[k];
      o.stream_staged = cands[k].stage;
      o.ctas_per_sm = cands[k].ctas;
      o.tile_cap = cands[k].tile_cap;
      o.configs_per_s = rate[k];
    };
    fill(bi, *best);
    if (n_tried) {
      const uint32_t cap = tried ? *n_tried : 0;
      *n_tried = static_cast<uint32_t>(cands.size());
      for (size_t k = 0; k < cands.size() && k < cap; ++k) fill(k, tried[k]);
    }
  });
}

sqsg_status sqsg_optimize(const sqsg_job* job, sqsg_run** run) { return run_jobs(job, 1, run, nullptr); }

sqsg_status sqsg_optimize_batch(const sqsg_job* jobs, uint32_t n_jobs, sqsg_run** runs) {
  return run_jobs(jobs, n_jobs, runs, nullptr);
}

sqsg_status sqsg_optimize_trace(const sqsg_job* job, sqsg_run** run, uint64_t capacity, uint64_t* count,
                                uint8_t* species, uint32_t* bonds, void* objective, uint64_t* id) {
  TraceOut t;
  t.capacity = capacity;
  t.count = count;
  t.species = species;
  t.bonds = bonds;
  t.objective = objective;
  t.id = id;
  if (capacity == 0) {
    set_error("trace capacity must be positive");
    return SQSG_ERR_INVALID_ARGUMENT;
  }
  sqsg_status s = run_jobs(job, 1, run, &t);
  if (s == SQSG_OK && count && *count > capacity) {
    set_error("trace capacity smaller than the number of evaluated configurations");
    return SQSG_ERR_CAPACITY;
  }
  return s;
}

uint64_t sqsg_run_count(const sqsg_run* run) { return run ? run->r.count : 0; }

sqsg_status sqsg_run_copy(const sqsg_run* run, uint64_t first, uint64_t n, void* objective, void* sub_objectives,
                          uint8_t* species, void* sro, uint64_t* id) {
  return guarded([&] {
    if (!run) throw std::invalid_argument("null run");
    const Run& r = run->r;
    if (first > r.count || n > r.count - first) throw std::out_of_range("record range out of bounds");
    size_t sp = 0, skk = 0;
    for (auto& p : r.parts) {
      sp += p.N;
      skk += static_cast<size_t>(p.S) * p.K * p.K;
    }
    if (objective) parallel_copy(objective, r.objective.data() + first * r.tsz, n * r.tsz);
    if (sub_objectives)
      parallel_copy(sub_objectives, r.sub_objective.data() + first * r.n_parts * r.tsz, n * r.n_parts * r.tsz);
    if (species) parallel_copy(species, r.species.data() + first * sp, n * sp);
    if (sro) parallel_copy(sro, r.sro.data() + first * skk * r.tsz, n * skk * r.tsz);
    if (id) parallel_copy(id, r.id.data() + first, n * 8);
  });
}

sqsg_status sqsg_run_statistics(const sqsg_run* run, sqsg_statistics* stats) {
  return guarded([&] {
    if (!run || !stats) throw std::invalid_argument("null pointer");
    *stats = run->r.stats;
  });
}

void sqsg_run_free(sqsg_run* run) { delete run; }

sqsg_status sqsg_run_levels(const sqsg_run* run, uint32_t* n, double* values, uint64_t* counts,
                            uint64_t* checksums) {
  return guarded([&] {
    if (!run || !n) throw std::invalid_argument("null pointer");
    const Run& r = run->r;
    const uint32_t cap = *n;
    *n = static_cast<uint32_t>(r.level_value.size());
    if (r.level_value.size() > cap) throw std::length_error("level capacity too small");
    for (size_t k = 0; k < r.level_value.size(); ++k) {
      if (values) values[k] = r.level_value[k];
      if (counts) counts[k] = r.level_count[k];
      if (checksums) checksums[k] = r.level_checksum[k];
    }
  });
}

sqsg_status sqsg_run_stages(const sqsg_run* run, uint64_t* ns, uint32_t* n) {
  return guarded([&] {
    if (!run || !n) throw std::invalid_argument("null pointer");
    const uint32_t cap = *n;
    *n = SQSG_STAGE_COUNT;
    if (cap < SQSG_STAGE_COUNT) throw std::length_error("stage capacity too small");
    if (ns)
      for (int k = 0; k < SQSG_STAGE_COUNT; ++k) ns[k] = run->r.stage_ns[k];
  });
}

sqsg_status sqsg_run_transfer(const sqsg_run* run, uint64_t* h2d_bytes, uint64_t* d2h_bytes) {
  return guarded([&] {
    if (!run) throw std::invalid_argument("null run");
    if (h2d_bytes) *h2d_bytes = run->r.h2d_bytes;
    if (d2h_bytes) *d2h_bytes = run->r.d2h_bytes;
  });
}

sqsg_status sqsg_run_info(const sqsg_run* run, uint64_t* candidates, int32_t* truncated, int32_t* levels_exact) {
  return guarded([&] {
    if (!run) throw std::invalid_argument("null run");
    if (candidates) *candidates = run->r.candidates;
    if (truncated) *truncated = run->r.truncated ? 1 : 0;
    if (levels_exact) *levels_exact = run->r.levels_exact ? 1 : 0;
  });
}



struct sqsg_server {
  ServerState s;
};

sqsg_status sqsg_server_create(const sqsg_server_options* options, sqsg_server** out) {
  return guarded([&] {
    if (!out) throw std::invalid_argument("null pointer");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      throw cuda_error("no CUDA device is available (the optimiser has no CPU path)");
    }
    sqsg_server_options opt{};
    if (options) opt = *options;
    if (opt.device < 0 || opt.device >= ndev) throw std::invalid_argument("invalid device ordinal");
    if (!opt.arena_bytes) {  // default: 16 GiB, at most a quarter of the free device memory
      CUDA_CHECK(cudaSetDevice(opt.device));
      size_t free_b = 0, total_b = 0;
      CUDA_CHECK(cudaMemGetInfo(&free_b, &total_b));
      opt.arena_bytes = std::min<uint64_t>(16ull << 30, free_b / 4);
    }
    if (!opt.max_jobs) opt.max_jobs = 256;
    if (!opt.default_max_results) opt.default_max_results = 1u << 16;
    auto srv = std::unique_ptr<sqsg_server, sqsg_status (*)(sqsg_server*)>(new sqsg_server, sqsg_server_destroy);
    ServerState& S = srv->s;
    S.opt = opt;
    S.device = opt.device;
    CUDA_CHECK(cudaSetDevice(S.device));
    CUDA_CHECK(cudaStreamCreateWithFlags(&S.copy, cudaStreamNonBlocking));
    const size_t optin = max_dynamic_smem(S.device);
    CUDA_CHECK(cudaMalloc(&S.d_ctl, kCtlBytes));
    CUDA_CHECK(cudaMemset(S.d_ctl, 0, kCtlBytes));
    CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&S.h_ctl), kCtlBytes, cudaHostAllocDefault));
    std::memset(S.h_ctl, 0, kCtlBytes);
    CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&S.h_yield), kBuckets * sizeof(uint32_t), cudaHostAllocDefault));
    CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&S.h_zero), kLevelSlots * sizeof(LevelSlot), cudaHostAllocDefault));
    std::memset(S.h_zero, 0, kLevelSlots * sizeof(LevelSlot));
    CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&S.h_ones), kOnesBytes, cudaHostAllocDefault));
    std::memset(S.h_ones, 0xff, kOnesBytes);
    CUDA_CHECK(cudaDeviceGetAttribute(&S.n_sm, cudaDevAttrMultiProcessorCount, S.device));
    if (S.n_sm > kMaxSm || S.n_sm <= kReservedSm) throw unsupported_error("unsupported SM count for the server");
    CUDA_CHECK(cudaMalloc(&S.d_owner, kMaxSm));
    CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&S.h_owner), kMaxSm, cudaHostAllocDefault));
    std::memset(S.h_owner, kNoOwner, kMaxSm);
    CUDA_CHECK(cudaMemcpy(S.d_owner, S.h_owner, kMaxSm, cudaMemcpyHostToDevice));
    // ring b: the largest dynamic shared memory at which 5 - b CTAs of its kernel fit on an SM
    configure_kernel(optin);
    for (int b = 0; b < kBuckets; ++b) {
      Ring& R = S.rings[b];
      R.kernel = kernel_of(kRingSpec[b].kind);
      auto fits = [&](size_t smem) {
        int nb = 0;
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, R.kernel, kBlock, smem));
        return nb;
      };
      const int want = kRingSpec[b].want;
      size_t lo = 0, hi = optin;  // largest smem in [0, optin] with fits(smem) >= want
      if (fits(hi) >= want) {
        lo = hi;
      } else {
        while (hi - lo > 16) {
          const size_t mid = (lo + hi) / 2 / 16 * 16;
          if (fits(mid) >= want)
            lo = mid;
          else
            hi = mid;
        }
      }
      R.smem = lo;
      R.per_sm = static_cast<uint32_t>(std::max(1, fits(lo)));
      for (auto& L : R.ls) {
        CUDA_CHECK(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
        CUDA_CHECK(cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming));
      }
      CUDA_CHECK(cudaMalloc(&S.d_ring[b], kRingCap * sizeof(Tile)));
      QueueCtl q{};
      q.capacity = static_cast<unsigned int>(kRingCap);
      q.idle_limit = kIdlePolls;
      q.ring = static_cast<unsigned int>(b);
      q.n_owner = static_cast<unsigned int>(S.n_sm);
      q.owner = S.d_owner;
      q.alive = S.d_alive(b);
      CUDA_CHECK(cudaMemcpy(S.q(b), &q, sizeof(q), cudaMemcpyHostToDevice));
    }
    CUDA_CHECK(cudaMalloc(&S.arena, S.opt.arena_bytes));
    S.free_list[0] = S.opt.arena_bytes;
    const size_t nslot = S.opt.max_jobs;
    CUDA_CHECK(cudaMalloc(&S.d_jobs, nslot * sizeof(JobDesc)));
    CUDA_CHECK(cudaMalloc(&S.d_counters, nslot * kNumCounters * 8));
    CUDA_CHECK(cudaMalloc(&S.d_levels, nslot * kLevelSlots * sizeof(LevelSlot)));
    CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&S.h_done), nslot * sizeof(uint32_t), cudaHostAllocMapped));
    CUDA_CHECK(cudaHostGetDevicePointer(reinterpret_cast<void**>(&S.d_done), S.h_done, 0));
    std::memset(S.h_done, 0, nslot * sizeof(uint32_t));
    S.slots.resize(nslot);
    S.slot_gen.assign(nslot, 0);
    S.worker = std::thread(server_loop, &S);
    const int finalizers = static_cast<int>(std::min<long long>(32, std::max<long long>(1, option(kOptServerFinalizers))));
    for (int k = 0; k < finalizers; ++k) S.finalizers.emplace_back(finalizer_loop, &S);
    *out = srv.release();
  });
}

sqsg_status sqsg_server_submit(sqsg_server* server, const sqsg_job* job, uint64_t* ticket) {
  return guarded([&] {
    if (!server || !job || !ticket) throw std::invalid_argument("null pointer");
    ServerState& S = server->s;
    if (job->device != S.device) throw std::invalid_argument("the job names another device than the server's");
    if (job->callback || job->cancel) throw std::invalid_argument("served jobs take no callback or cancel flag");
    auto J = std::make_unique<ServerJob>();
    J->pj = prepare(*job, 0);
    if (J->pj.chain) throw unsupported_error("the rapidrand debug mode runs through sqsg_optimize, not the server");
    J->t_submit = now_ns();
    const size_t need = J->pj.desc.smem_bytes;
    const int kind = kind_of(J->pj.desc);
    J->bucket = -1;
    for (int b = 0; b < kBuckets; ++b)  // rings of one kernel are ordered by falling occupancy
      if (kRingSpec[b].kind == kind && need <= S.rings[b].smem) {
        J->bucket = b;
        break;
      }
    // a bit-mask job may run the general path as well, and every lattice job the eight-species kernel
    const int other = kind == kKindMask ? kKindWide : (is_lattice_kind(kind) && kind != kKindLatW ? kKindLat : -1);
    if (J->bucket < 0 && other >= 0)
      for (int b = 0; b < kBuckets; ++b)
        if (kRingSpec[b].kind == other && need <= S.rings[b].smem) {
          J->bucket = b;
          break;
        }
    if (J->bucket < 0) throw unsupported_error("the job needs more shared memory per CTA than this device offers");
    J->user_capacity = job->max_results != 0;
    J->capacity = job->max_results ? job->max_results : S.opt.default_max_results;
    J->cost = config_cost(J->pj);
    make_tiles(J->pj, 0, J->tiles, std::max<uint64_t>(1, static_cast<uint64_t>(kTilePairs / J->cost)));
    if (J->tiles.size() > kRingCap) throw unsupported_error("the job has more tiles than the ring holds");
    J->cum.assign(J->tiles.size() + 1, 0);
    for (size_t k = 0; k < J->tiles.size(); ++k) J->cum[k + 1] = J->cum[k] + J->tiles[k].count;
    if (job_footprint(*J) > S.opt.arena_bytes)
      throw std::length_error("the job's device footprint exceeds the server's arena; lower max_results");
    std::lock_guard<std::mutex> l(S.m);
    if (!S.broken.empty()) throw cuda_error("the server stopped after a device error: " + S.broken);
    J->ticket = S.next_ticket++;
    *ticket = J->ticket;
    S.stats.submitted++;
    if (J->tiles.empty()) {  // nothing to evaluate: an empty result
      Run r;
      r.prec = J->pj.prec;
      r.n_parts = J->pj.desc.n_parts;
      r.parts = J->pj.parts;
      r.tsz = J->pj.tsz;
      r.stats.best_objective = std::numeric_limits<double>::infinity();
      S.finished.emplace(J->ticket, std::move(r));
      S.stats.completed++;
      S.cv_done.notify_all();
      return;
    }
    S.pending.push_back(std::move(J));
    S.cv_work.notify_one();
  });
}

sqsg_status sqsg_server_wait(sqsg_server* server, uint64_t ticket, int64_t timeout_us, sqsg_run** run) {
  return guarded([&] {
    if (!server || !run) throw std::invalid_argument("null pointer");
    ServerState& S = server->s;
    std::unique_lock<std::mutex> l(S.m);
    auto ready = [&] { return S.finished.count(ticket) || S.failed.count(ticket); };
    if (timeout_us < 0)
      S.cv_done.wait(l, ready);
    else if (!S.cv_done.wait_for(l, std::chrono::microseconds(timeout_us), ready))
      throw timeout_error("the job has not finished yet");
    auto f = S.failed.find(ticket);
    if (f != S.failed.end()) {
      const auto err = f->second;
      S.failed.erase(f);
      throw cuda_error(err.second);
    }
    auto it = S.finished.find(ticket);
    *run = new sqsg_run{std::move(it->second)};
    S.finished.erase(it);
  });
}

sqsg_status sqsg_server_stats(sqsg_server* server, sqsg_server_counters* stats) {
  return guarded([&] {
    if (!server || !stats) throw std::invalid_argument("null pointer");
    ServerState& S = server->s;
    std::lock_guard<std::mutex> l(S.m);
    *stats = S.stats;
    stats->pending = S.pending.size();
    uint64_t active = 0;
    for (auto& x : S.slots) active += x ? 1 : 0;
    stats->active = active;
    size_t free_bytes = 0;
    for (auto& [o, n] : S.free_list) free_bytes += n;
    stats->arena_free_bytes = free_bytes;
  });
}

sqsg_status sqsg_server_running(sqsg_server* server, uint32_t* launches) {
  return guarded([&] {
    if (!server || !launches) throw std::invalid_argument("null pointer");
    ServerState& S = server->s;
    std::lock_guard<std::mutex> l(S.m);
    uint32_t n = 0;
    for (auto& R : S.rings)
      for (auto& L : R.ls) n += L.busy ? 1u : 0u;
    *launches = n;
  });
}

sqsg_status sqsg_server_destroy(sqsg_server* server) {
  if (!server) return SQSG_OK;
  ServerState& S = server->s;
  {
    std::lock_guard<std::mutex> l(S.m);
    S.stop = true;
    S.cv_work.notify_all();
    S.cv_fin.notify_all();
  }
  if (S.worker.joinable()) S.worker.join();
  for (auto& t : S.finalizers)
    if (t.joinable()) t.join();
  cudaSetDevice(S.device);
  // every CTA leaves at its next claim: no tile is started after this
  if (S.d_ctl && S.h_yield && S.copy) {
    if (S.d_owner && S.h_owner) {
      std::memset(S.h_owner, kNoOwner, kMaxSm);
      cudaMemcpyAsync(S.d_owner, S.h_owner, kMaxSm, cudaMemcpyHostToDevice, S.copy);
    }
    for (int b = 0; b < kBuckets; ++b) {
      S.h_yield[b] = ~0u;
      cudaMemcpyAsync(&S.q(b)->yield, &S.h_yield[b], sizeof(uint32_t), cudaMemcpyHostToDevice, S.copy);
    }
    cudaStreamSynchronize(S.copy);
  }
  for (auto& R : S.rings)
    for (auto& L : R.ls)
      if (L.stream) cudaStreamSynchronize(L.stream);
  for (int b = 0; b < kBuckets; ++b) {
    for (auto& L : S.rings[b].ls) {
      if (L.stream) cudaStreamDestroy(L.stream);
      if (L.done) cudaEventDestroy(L.done);
    }
    if (S.d_ring[b]) cudaFree(S.d_ring[b]);
  }
  if (S.copy) cudaStreamDestroy(S.copy);
  if (S.arena) cudaFree(S.arena);
  if (S.d_jobs) cudaFree(S.d_jobs);
  if (S.d_counters) cudaFree(S.d_counters);
  if (S.d_levels) cudaFree(S.d_levels);
  if (S.d_ctl) cudaFree(S.d_ctl);
  if (S.h_ctl) cudaFreeHost(S.h_ctl);
  if (S.h_yield) cudaFreeHost(S.h_yield);
  if (S.h_zero) cudaFreeHost(S.h_zero);
  if (S.h_ones) cudaFreeHost(S.h_ones);
  if (S.d_owner) cudaFree(S.d_owner);
  if (S.h_owner) cudaFreeHost(S.h_owner);
  if (S.h_done) cudaFreeHost(S.h_done);
  delete server;
  return SQSG_OK;
}

}  // extern "C"
