// Allocation-free entry point: sqsg_optimize_levels_noalloc.
//
// Some callers cannot allocate device memory: code running inside a framework that owns the whole
// device budget through its own pool, processes whose memory is capped at start-up, and hosts that
// must not call cudaMalloc/cudaFree once work has started. For them this entry point runs the same
// engine kernel as sqsg_optimize, but every device-side buffer it needs (job descriptor, counters,
// objective-level table, tile list and the job's staged data) lives in one file-scope
// `static __device__` array of kScratchBytes, and the host side stages through a fixed static buffer.
// It calls no cudaMalloc, cudaFree, cudaHostAlloc, stream/event creation or other allocating routine.
//
// What it returns: the keep+1 best distinct objectives with their exact counts and id checksums and
// the run statistics — the same values sqsg_run_levels / sqsg_run_statistics report for the same job —
// but no configuration records (those need buffers sized by the result set).
//
// Limits: the staged job data must fit kBlobBytes and the tile list kMaxTiles (errors otherwise);
// no progress callback and no cancellation.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>

#include "engine.cuh"
#include "permutation.h"
#include "sqsg_internal.h"
#include "tiles.h"

namespace sqsg {

__global__ void __launch_bounds__(kBlock, kMinBlocks)
    sqsg_engine(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done);

namespace noalloc {

// Scratch layout (byte offsets inside the device array).
constexpr size_t kDescOff = 0;                                   // JobDesc
constexpr size_t kCountersOff = 4096;                            // kNumCounters u64
constexpr size_t kQueueOff = kCountersOff + 256;                 // QueueCtl
constexpr size_t kStatusOff = kQueueOff + 64;                    // u64 device status
constexpr size_t kLevelsOff = 8192;                              // kLevelSlots LevelSlot
constexpr size_t kTilesOff = kLevelsOff + kLevelSlots * sizeof(LevelSlot);
constexpr size_t kMaxTiles = 16448;
constexpr size_t kBlobOff = kTilesOff + kMaxTiles * sizeof(Tile);
constexpr size_t kBlobBytes = 3u << 20;                          // staged job data, at most 3 MiB
constexpr size_t kScratchBytes = kBlobOff + kBlobBytes;          // about 3.6 MiB in total

static_assert(sizeof(JobDesc) <= kCountersOff, "descriptor slot too small");
static_assert(kBlobOff % 256 == 0, "blob must stay 256-byte aligned");

// The device scratch. In host code `g_scratch` is only a handle for the runtime: its device address
// comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Host staging for the job blob and the tile list (fixed, reused by every call; guarded by g_mutex).
static unsigned char g_stage_blob[kBlobBytes];
static Tile g_stage_tiles[kMaxTiles];
static std::mutex g_mutex;

constexpr int kMaxDevices = 64;
static unsigned char* g_dev_ptr[kMaxDevices];

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
static inline uint32_t site_off(uint32_t x) { return (x >> 2) * (kBlock * 4) + (x & 3); }

static unsigned long long ord_bits(double x) {
  unsigned long long b;
  std::memcpy(&b, &x, 8);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

static double from_ord(unsigned long long u) {
  unsigned long long b = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
  double x;
  std::memcpy(&x, &b, 8);
  return x;
}

// Errors travel as (status, static message) pairs; nothing on this path throws or allocates.
struct Err {
  sqsg_status status;
  const char* msg;
};
constexpr Err kOk{SQSG_OK, nullptr};

#define NA_FAIL(st, m) \
  do {                 \
    return Err{st, m}; \
  } while (0)
#define NA_CUDA(expr, m)                            \
  do {                                              \
    if ((expr) != cudaSuccess) NA_FAIL(SQSG_ERR_CUDA, m); \
  } while (0)
#define NA_TRY(expr)             \
  do {                           \
    const Err e__ = (expr);      \
    if (e__.status != SQSG_OK) return e__; \
  } while (0)

// Device address of g_scratch on the current device, looked up on the first call per device.
static Err scratch_for(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "device ordinal out of range");
  if (!g_dev_ptr[device]) {
    void* p = nullptr;
    NA_CUDA(cudaGetSymbolAddress(&p, g_scratch), "cudaGetSymbolAddress(g_scratch) failed");
    g_dev_ptr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_dev_ptr[device];
  return kOk;
}

// Lays out one job exactly like the heap-based preparation of sqsg_optimize (same staged sections,
// shared-memory layout and tile decomposition) but writes into the static staging buffers.
static Err prepare(const sqsg_job& job, JobDesc& d, size_t& blob_size, size_t& n_tiles) {
  if (job.prec != SQSG_PREC_SINGLE && job.prec != SQSG_PREC_DOUBLE) NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "invalid prec");
  if (job.iteration_mode != SQSG_ITERATION_RANDOM && job.iteration_mode != SQSG_ITERATION_SYSTEMATIC)
    NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "invalid iteration mode");
  if (job.sublattice_mode != SQSG_SUBLATTICE_INTERACT && job.sublattice_mode != SQSG_SUBLATTICE_SPLIT)
    NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "invalid sublattice mode");
  if (!job.sublattices || job.n_sublattices == 0) NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "no sublattices");
  if (job.sublattice_mode == SQSG_SUBLATTICE_INTERACT && job.n_sublattices != 1)
    NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "interact mode takes one optimised structure");
  if (job.n_sublattices > static_cast<uint32_t>(kMaxParts)) NA_FAIL(SQSG_ERR_UNSUPPORTED, "more than 8 sublattices");
  const bool systematic = job.iteration_mode == SQSG_ITERATION_SYSTEMATIC;
  if (systematic && job.sublattice_mode == SQSG_SUBLATTICE_SPLIT)
    NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "no exhaustive search on multiple sublattices in split mode");
  if (job.keep == 0) NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "keep must be greater than 0");
  if (job.keep > 31) NA_FAIL(SQSG_ERR_UNSUPPORTED, "keep > 31 is not supported");
  const size_t tsz = job.prec == SQSG_PREC_DOUBLE ? 8 : 4;
  std::memset(&d, 0, sizeof(d));
  d.prec = static_cast<uint32_t>(job.prec);
  d.mode = systematic ? 1 : 0;
  d.n_parts = job.n_sublattices;
  d.keep = static_cast<uint32_t>(job.keep);
  d.kw = 1;
  size_t smem = 0;
  blob_size = 0;
  uint64_t total = 0;
  for (uint32_t p = 0; p < job.n_sublattices; ++p) {
    const sqsg_sublattice& sl = job.sublattices[p];
    PartDesc& P = d.parts[p];
    if (sl.n_sites == 0) NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "empty structure");
    if (sl.n_species == 0 || sl.n_shells == 0) NA_FAIL(SQSG_ERR_OUT_OF_RANGE, "no coordination shells selected");
    if (sl.n_species > static_cast<uint32_t>(kMaxSpecies)) NA_FAIL(SQSG_ERR_UNSUPPORTED, "more than 8 species");
    if (sl.n_shells > 255) NA_FAIL(SQSG_ERR_UNSUPPORTED, "more than 255 shells");
    if (!sl.species || !sl.prefactors || !sl.pair_weights || !sl.target || (sl.n_pairs && !sl.pairs))
      NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "null array in sublattice");
    if (sl.n_windows == 0 || !sl.windows) NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "no shuffle window");
    if (sl.n_windows > static_cast<uint32_t>(kMaxWindows)) NA_FAIL(SQSG_ERR_UNSUPPORTED, "more than 16 windows");
    for (uint32_t x = 0; x < sl.n_sites; ++x)
      if (sl.species[x] >= sl.n_species) NA_FAIL(SQSG_ERR_OUT_OF_RANGE, "packed species index >= n_species");
    for (uint32_t w = 0; w < sl.n_windows; ++w) {
      if (sl.windows[2 * w] >= sl.windows[2 * w + 1] || sl.windows[2 * w + 1] > sl.n_sites)
        NA_FAIL(SQSG_ERR_OUT_OF_RANGE, "invalid shuffle window");
      if (w > 0 && sl.windows[2 * w] < sl.windows[2 * w - 1]) NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "overlapping windows");
    }
    if (systematic && sl.n_windows != 1) NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "systematic mode allows one sublattice");
    const uint32_t N = sl.n_sites, S = sl.n_shells, K = sl.n_species;
    P.n_sites = N;
    P.n_species = K;
    P.n_shells = S;
    P.n_windows = sl.n_windows;
    P.hw = (K + 1) / 2;
    if (K > 4) d.kw = 2;
    for (uint32_t e = 0; e < sl.n_pairs; ++e) {
      const uint32_t i = sl.pairs[3 * e], j = sl.pairs[3 * e + 1], s = sl.pairs[3 * e + 2];
      if (i >= N || j >= N) NA_FAIL(SQSG_ERR_OUT_OF_RANGE, "pair index out of range");
      if (s >= S) NA_FAIL(SQSG_ERR_OUT_OF_RANGE, "pair shell index out of range");
      if (i == j) NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "pair with i == j");
    }
    // count the stream words: groups of <= kMaxGroup neighbours per (shell, site)
    const bool narrow = site_off(N ? N - 1 : 0) < 0x10000u;
    P.stream_narrow = narrow ? 1u : 0u;
    size_t words = 0;
    for (uint32_t s = 0; s < S; ++s) {
      uint64_t in_shell = 0;
      for (uint32_t i = 0; i < N; ++i) {
        uint32_t cnt = 0;
        for (uint32_t e = 0; e < sl.n_pairs; ++e)
          if (sl.pairs[3 * e + 2] == s && std::min(sl.pairs[3 * e], sl.pairs[3 * e + 1]) == i) ++cnt;
        in_shell += cnt;
        for (uint32_t left = cnt; left > 0;) {  // the same groups as the regular entry point
          const uint32_t g = std::min<uint32_t>(left, kMaxGroup);
          words += narrow ? 1ull + (g + 1) / 2 : 2ull + g;
          left -= g;
        }
      }
      if (in_shell > 0xffffu) NA_FAIL(SQSG_ERR_UNSUPPORTED, "a shell holds more than 65535 pairs");
    }
    const size_t skk = static_cast<size_t>(S) * K * K;
    size_t off = 0;
    P.cube_off = 0;
    off = align_up(3 * skk * tsz, 16);
    P.win_off = static_cast<uint32_t>(off);
    off = align_up(off + 8ull * sl.n_windows, 16);
    P.species_off = static_cast<uint32_t>(off);
    off = align_up(off + N, 16);
    P.static_bytes = static_cast<uint32_t>(off);  // staged; the stream after it is read from the blob
    P.stream_off = static_cast<uint32_t>(off);
    P.stream_global = 1;
    const size_t section = align_up(off + 4ull * words, 16);
    P.blob_off = static_cast<uint32_t>(blob_size);
    if (blob_size + section > kBlobBytes) NA_FAIL(SQSG_ERR_CAPACITY, "job data exceeds the 3 MiB static staging area");
    P.stream_words = static_cast<uint32_t>(words);
    // fill the staged section
    unsigned char* base = g_stage_blob + blob_size;
    std::memset(base, 0, section);
    std::memcpy(base + P.cube_off, sl.prefactors, skk * tsz);
    std::memcpy(base + P.cube_off + skk * tsz, sl.pair_weights, skk * tsz);
    std::memcpy(base + P.cube_off + 2 * skk * tsz, sl.target, skk * tsz);
    std::memcpy(base + P.win_off, sl.windows, 8ull * sl.n_windows);
    uint32_t* st = reinterpret_cast<uint32_t*>(base + P.stream_off);
    size_t w = 0;
    for (uint32_t s = 0; s < S; ++s)
      for (uint32_t i = 0; i < N; ++i) {
        uint32_t in_group = 0;
        size_t hdr = 0;
        for (uint32_t e = 0; e < sl.n_pairs; ++e) {
          const uint32_t a = sl.pairs[3 * e], b = sl.pairs[3 * e + 1];
          if (sl.pairs[3 * e + 2] != s || std::min(a, b) != i) continue;
          if (in_group == 0 || in_group == static_cast<uint32_t>(kMaxGroup)) {
            hdr = w;
            st[w++] = 0;
            if (!narrow) st[w++] = site_off(i);
            in_group = 0;
          }
          const uint32_t jo = site_off(std::max(a, b));
          if (!narrow)
            st[w++] = jo;
          else if (in_group % 2 == 0)
            st[w++] = jo;
          else
            st[w - 1] |= jo << 16;
          ++in_group;
          st[hdr] = narrow ? (site_off(i) | (s << 16) | (in_group << 24)) : (s | (in_group << 8));
        }
      }
    for (uint32_t x = 0; x < N; ++x) base[P.species_off + x] = static_cast<unsigned char>(sl.species[x] << 3);
    blob_size += section;
    P.smem_off = static_cast<uint32_t>(smem);
    P.col_off = static_cast<uint32_t>(off);
    off += static_cast<size_t>((N + 3) / 4) * kBlock * 4;
    P.hist_off = static_cast<uint32_t>(off);
    off += static_cast<size_t>(S) * K * P.hw * kBlock * 4;
    smem += align_up(off, 16);
    if (systematic) {
      const uint32_t lo = sl.windows[0], hi = sl.windows[1];
      uint32_t counts[256] = {0};
      for (uint32_t x = lo; x < hi; ++x) counts[sl.species[x]]++;
      uint32_t k = 0, dense[kMaxSpecies];
      for (uint32_t v = 0; v < 256; ++v)
        if (counts[v]) {
          if (k >= static_cast<uint32_t>(kMaxSpecies)) NA_FAIL(SQSG_ERR_UNSUPPORTED, "more than 8 species in the window");
          P.unrank_rev[k] = static_cast<uint8_t>(v);
          P.unrank_hist[k] = counts[v];
          dense[k++] = counts[v];
        }
      P.unrank_k = k;
      if (!num_permutations_counts(dense, static_cast<int>(k), &total))
        NA_FAIL(SQSG_ERR_OUT_OF_RANGE, "the number of permutations does not fit in 64 bits");
    }
  }
  if (!systematic) total = job.iterations;
  d.total = total;
  d.smem_bytes = static_cast<uint32_t>(smem);
  d.record_bytes = 16;
  d.capacity = 0;  // no records: the level table carries the result
  if (job.has_seed) {
    d.seed = job.seed;
  } else {
    unsigned long long t = static_cast<unsigned long long>(std::chrono::steady_clock::now().time_since_epoch().count());
    d.seed = t * 0x9e3779b97f4a7c15ull;
  }
  if (job.range_first > total) NA_FAIL(SQSG_ERR_OUT_OF_RANGE, "range_first beyond the configuration space");
  const uint64_t count = job.range_count ? job.range_count : total - job.range_first;
  if (count > total - job.range_first) NA_FAIL(SQSG_ERR_OUT_OF_RANGE, "range beyond the configuration space");
  d.trace_base = job.range_first + (systematic ? 1 : 0);
  // tiles: the same decomposition as sqsg_optimize (tiles.h)
  n_tiles = 0;
  bool too_many = false;
  for_each_tile(job.range_first, count, systematic, [&](const Tile& t) -> bool {
    if (n_tiles >= kMaxTiles) {
      too_many = true;
      return false;  // stop at once: a job of 1e18 configurations has ~1e11 tiles
    }
    g_stage_tiles[n_tiles++] = t;
    return true;
  });
  if (too_many) NA_FAIL(SQSG_ERR_CAPACITY, "the job needs more tiles than the static tile list holds");
  return kOk;
}

// One call: stage, launch the engine on the static scratch, read back the level table.
static Err run(const sqsg_job& job, void* stream, uint32_t* n_levels, double* values, uint64_t* counts,
               uint64_t* checksums, sqsg_statistics* stats) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    NA_FAIL(SQSG_ERR_CUDA, "no CUDA device is available (the optimiser has no CPU path)");
  }
  if (job.device < 0 || job.device >= ndev) NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "invalid device ordinal");
  NA_CUDA(cudaSetDevice(job.device), "cudaSetDevice failed");
  unsigned char* dev = nullptr;
  NA_TRY(scratch_for(job.device, &dev));
  JobDesc d;
  size_t blob_size = 0, n_tiles = 0;
  NA_TRY(prepare(job, d, blob_size, n_tiles));
  int optin = 0;
  NA_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, job.device), "attribute query");
  cudaFuncAttributes attr{};
  NA_CUDA(cudaFuncGetAttributes(&attr, sqsg_engine), "cudaFuncGetAttributes failed");
  if (d.smem_bytes > static_cast<size_t>(optin) - attr.sharedSizeBytes)
    NA_FAIL(SQSG_ERR_UNSUPPORTED, "the job needs more shared memory per CTA than the device offers");
  // The kernel attribute is process-wide and other entry points rely on it only growing: raise it
  // when this job needs more, never lower it.
  if (static_cast<int>(d.smem_bytes) > attr.maxDynamicSharedSizeBytes)
    NA_CUDA(cudaFuncSetAttribute(sqsg_engine, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(d.smem_bytes)),
            "cudaFuncSetAttribute failed");
  d.blob = dev + kBlobOff;
  d.records = dev + kBlobOff;  // never written: capacity is 0
  d.counters = reinterpret_cast<unsigned long long*>(dev + kCountersOff);
  d.levels = reinterpret_cast<LevelSlot*>(dev + kLevelsOff);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the array keeps the previous call's contents: reset counters, queue, status and level table
  unsigned long long init[kNumCounters] = {0};
  const double maxv = job.prec == SQSG_PREC_DOUBLE ? std::numeric_limits<double>::max()
                                                   : static_cast<double>(std::numeric_limits<float>::max());
  init[kThreshold] = ord_bits(maxv);
  init[kBest] = ord_bits(std::numeric_limits<double>::infinity());
  NA_CUDA(cudaMemcpyAsync(dev + kDescOff, &d, sizeof(d), cudaMemcpyHostToDevice, s), "descriptor upload");
  NA_CUDA(cudaMemcpyAsync(dev + kCountersOff, init, sizeof(init), cudaMemcpyHostToDevice, s), "counter upload");
  NA_CUDA(cudaMemsetAsync(dev + kQueueOff, 0, sizeof(QueueCtl), s), "queue reset");
  NA_CUDA(cudaMemsetAsync(dev + kStatusOff, 0, 8, s), "status reset");
  NA_CUDA(cudaMemsetAsync(dev + kLevelsOff, 0, kLevelSlots * sizeof(LevelSlot), s), "level reset");
  if (blob_size) NA_CUDA(cudaMemcpyAsync(dev + kBlobOff, g_stage_blob, blob_size, cudaMemcpyHostToDevice, s), "blob upload");
  if (n_tiles)
    NA_CUDA(cudaMemcpyAsync(dev + kTilesOff, g_stage_tiles, n_tiles * sizeof(Tile), cudaMemcpyHostToDevice, s),
            "tile upload");
  int per_sm = 0, sms = 0;
  NA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sqsg_engine, kBlock, d.smem_bytes), "occupancy");
  NA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, job.device), "attribute query");
  if (per_sm <= 0) NA_FAIL(SQSG_ERR_UNSUPPORTED, "the job does not fit on one SM");
  const auto t0 = std::chrono::steady_clock::now();
  if (n_tiles) {
    const size_t grid = std::max<size_t>(1, std::min<size_t>(n_tiles, static_cast<size_t>(per_sm) * sms));
    sqsg_engine<<<static_cast<uint32_t>(grid), kBlock, d.smem_bytes, s>>>(
        reinterpret_cast<const JobDesc*>(dev + kDescOff), reinterpret_cast<const Tile*>(dev + kTilesOff),
        static_cast<uint32_t>(n_tiles), reinterpret_cast<QueueCtl*>(dev + kQueueOff), nullptr,
        reinterpret_cast<unsigned long long*>(dev + kStatusOff), nullptr);
    NA_CUDA(cudaGetLastError(), "engine launch failed");
  }
  static LevelSlot lv[kLevelSlots];  // static: guarded by g_mutex, keeps 96 KiB off the caller's stack
  unsigned long long cnt[kNumCounters], status = 0;
  NA_CUDA(cudaMemcpyAsync(lv, dev + kLevelsOff, sizeof(lv), cudaMemcpyDeviceToHost, s), "level download");
  NA_CUDA(cudaMemcpyAsync(cnt, dev + kCountersOff, sizeof(cnt), cudaMemcpyDeviceToHost, s), "counter download");
  NA_CUDA(cudaMemcpyAsync(&status, dev + kStatusOff, 8, cudaMemcpyDeviceToHost, s), "status download");
  NA_CUDA(cudaStreamSynchronize(s), "engine run failed");
  const auto t1 = std::chrono::steady_clock::now();
  if (status == kErrStageTimeout) NA_FAIL(SQSG_ERR_TIMEOUT, "shared-memory staging wait timed out on the device");
  if (status) NA_FAIL(SQSG_ERR_CUDA, "device error");
  // the keep+1 smallest objective keys, by insertion into a fixed array
  const uint32_t want = static_cast<uint32_t>(job.keep + 1);
  LevelSlot best[32];
  uint32_t nb = 0;
  for (int k = 0; k < kLevelSlots; ++k) {
    if (!lv[k].key) continue;
    uint32_t pos = nb;
    while (pos > 0 && best[pos - 1].key > lv[k].key) --pos;
    if (pos >= want) continue;
    const uint32_t last = std::min(nb, want - 1);
    for (uint32_t m = last; m > pos; --m) best[m] = best[m - 1];
    best[pos] = lv[k];
    nb = std::min(nb + 1, want);
  }
  const uint32_t cap = *n_levels;
  *n_levels = nb;
  for (uint32_t k = 0; k < std::min(nb, cap); ++k) {
    if (values) values[k] = from_ord(best[k].key);
    if (counts) counts[k] = best[k].count;
    if (checksums) checksums[k] = static_cast<uint64_t>(best[k].sum_a) | (static_cast<uint64_t>(best[k].sum_b) << 32);
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->finished = cnt[kFinished];
    stats->best_objective = nb ? from_ord(best[0].key) : std::numeric_limits<double>::infinity();
    const uint64_t ns = static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count());
    stats->timings_ns[SQSG_TIMING_TOTAL] = ns;
    stats->timings_ns[SQSG_TIMING_LOOP] = ns;
  }
  if (cnt[kLevelOverflow]) NA_FAIL(SQSG_ERR_CAPACITY, "the objective-level table overflowed; levels are incomplete");
  if (nb > cap) NA_FAIL(SQSG_ERR_CAPACITY, "level capacity too small");
  return kOk;
}

}  // namespace noalloc
}  // namespace sqsg

using namespace sqsg;
using namespace sqsg::noalloc;

extern "C" {

sqsg_status sqsg_optimize_levels_noalloc(const sqsg_job* job, void* stream, uint32_t* n_levels, double* values,
                                         uint64_t* counts, uint64_t* checksums, sqsg_statistics* stats, char* err,
                                         size_t err_len) {
  auto report = [&](sqsg_status s, const char* msg) {
    if (err && err_len) {
      std::snprintf(err, err_len, "%s", msg);
    }
    return s;
  };
  if (!job || !n_levels) return report(SQSG_ERR_INVALID_ARGUMENT, "null pointer");
  std::lock_guard<std::mutex> lock(g_mutex);
  const Err e = run(*job, stream, n_levels, values, counts, checksums, stats);
  return report(e.status, e.msg ? e.msg : "");
}

}  // extern "C"
