// Allocation-free entry point: sqsg_optimize_levels_noalloc.
//
// Some callers cannot allocate device memory: code running inside a framework that owns the whole
// device budget through its own pool, processes whose device memory is capped once work starts, and
// hosts that must not call cudaMalloc/cudaFree while other work runs. For them this entry point runs
// the same engine as sqsg_optimize, prepared by the same host code (prepare.cu), but every device-side
// buffer it needs (job descriptor, counters, objective-level table, tile list and the job's staged
// data) lives in one file-scope `static __device__` array of kScratchBytes. It calls no cudaMalloc,
// cudaFree, cudaMallocAsync, cudaHostAlloc, stream/event creation or other routine that allocates
// device or pinned memory; the host-side preparation uses ordinary host memory like sqsg_optimize.
//
// What it returns: the keep+1 best distinct objectives with their exact counts and id checksums —
// the values sqsg_run_levels reports for the same job — and the run statistics, but no configuration
// records (those need device buffers sized by the result set).
//
// A job whose level table overflows runs again from a tighter threshold (at most kMaxPasses passes).
// Limits: the staged job data must fit kBlobBytes and the tile list kMaxTiles (errors otherwise);
// no progress callback and no cancellation.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include "engine.cuh"
#include "kernels.h"
#include "prepare.h"
#include "sqsg_internal.h"
#include "tiles.h"

namespace sqsg {
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

static std::mutex g_mutex;  // serialises the calls of this process (they share g_scratch)

constexpr int kMaxDevices = 64;
static unsigned char* g_dev_ptr[kMaxDevices];

// Errors travel as (status, message) pairs out of this file's functions.
struct Err {
  sqsg_status status;
  std::string msg;
};

#define NA_FAIL(st, m) \
  do {                 \
    return Err{st, m}; \
  } while (0)
#define NA_CUDA(expr, m)                                                                   \
  do {                                                                                     \
    const cudaError_t e__ = (expr);                                                        \
    if (e__ != cudaSuccess) NA_FAIL(SQSG_ERR_CUDA, std::string(m) + ": " + cudaGetErrorString(e__)); \
  } while (0)
#define NA_TRY(expr)                       \
  do {                                     \
    Err e__ = (expr);                      \
    if (e__.status != SQSG_OK) return e__; \
  } while (0)

static Err ok() { return Err{SQSG_OK, std::string()}; }

// Device address of g_scratch on the current device, looked up on the first call per device.
static Err scratch_for(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) NA_FAIL(SQSG_ERR_INVALID_ARGUMENT, "device ordinal out of range");
  if (!g_dev_ptr[device]) {
    void* p = nullptr;
    NA_CUDA(cudaGetSymbolAddress(&p, g_scratch), "cudaGetSymbolAddress(g_scratch)");
    g_dev_ptr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_dev_ptr[device];
  return ok();
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
  // the same preparation and tiles as sqsg_optimize (host memory only)
  PreparedJob pj;
  std::vector<Tile> tiles;
  bool too_many = false;
  const sqsg_status ps = guarded([&] {
    pj = prepare(job, 0);
    // the same tiles as sqsg_optimize, stopping as soon as the static list is exceeded
    for_each_tile(pj.range_first, pj.range_count, pj.systematic, [&](Tile t) -> bool {
      if (tiles.size() >= kMaxTiles) {
        too_many = true;
        return false;
      }
      tiles.push_back(t);
      return true;
    });
  });
  if (ps != SQSG_OK) {
    char msg[512];
    sqsg_last_error(msg, sizeof(msg));
    NA_FAIL(ps, msg);
  }
  if (pj.chain) NA_FAIL(SQSG_ERR_UNSUPPORTED, "the rapidrand debug mode runs through sqsg_optimize");
  if (pj.blob.size() > kBlobBytes) NA_FAIL(SQSG_ERR_CAPACITY, "job data exceeds the 3 MiB static staging area");
  if (too_many) NA_FAIL(SQSG_ERR_CAPACITY, "the job needs more tiles than the static tile list holds");
  JobDesc d = pj.desc;
  const size_t n_tiles = tiles.size();
  // the kernel sqsg_optimize would launch for this job
  const EngineKernel kernel = kernel_of(kind_of(d));
  int optin = 0;
  NA_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, job.device), "attribute query");
  cudaFuncAttributes attr{};
  NA_CUDA(cudaFuncGetAttributes(&attr, kernel), "cudaFuncGetAttributes");
  if (d.smem_bytes > static_cast<size_t>(optin) - attr.sharedSizeBytes)
    NA_FAIL(SQSG_ERR_UNSUPPORTED, "the job needs more shared memory per CTA than the device offers");
  // The attribute is per device and shared with the other entry points: one helper raises it
  // (never lowers it) under one lock for every caller.
  if (raise_dynamic_smem(reinterpret_cast<const void*>(kernel), d.smem_bytes) != 0)
    NA_FAIL(SQSG_ERR_CUDA, "cudaFuncSetAttribute failed");
  d.blob = dev + kBlobOff;
  d.records = dev + kBlobOff;  // never written: capacity is 0
  d.capacity = 0;              // no records: the level table carries the result
  d.counters = reinterpret_cast<unsigned long long*>(dev + kCountersOff);
  d.levels = reinterpret_cast<LevelSlot*>(dev + kLevelsOff);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int per_sm = 0, sms = 0;
  NA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, d.smem_bytes), "occupancy");
  NA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, job.device), "attribute query");
  if (per_sm <= 0) NA_FAIL(SQSG_ERR_UNSUPPORTED, "the job does not fit on one SM");
  const double maxv = pj.prec == SQSG_PREC_DOUBLE ? std::numeric_limits<double>::max()
                                                   : static_cast<double>(std::numeric_limits<float>::max());
  static LevelSlot lv[kLevelSlots];  // static: guarded by g_mutex, keeps 96 KiB off the caller's stack
  unsigned long long cnt[kNumCounters];
  // One pass over every tile: the array keeps the previous pass's contents, so counters, queue,
  // status and level table are reset first; `threshold` is the ordered key the table starts from.
  auto pass = [&](unsigned long long threshold) -> Err {
    unsigned long long init[kNumCounters] = {0};
    init[kThreshold] = threshold;
    init[kBest] = ord_bits(std::numeric_limits<double>::infinity());
    NA_CUDA(cudaMemcpyAsync(dev + kDescOff, &d, sizeof(d), cudaMemcpyHostToDevice, s), "descriptor upload");
    NA_CUDA(cudaMemcpyAsync(dev + kCountersOff, init, sizeof(init), cudaMemcpyHostToDevice, s), "counter upload");
    NA_CUDA(cudaMemsetAsync(dev + kQueueOff, 0, sizeof(QueueCtl), s), "queue reset");
    NA_CUDA(cudaMemsetAsync(dev + kStatusOff, 0, 8, s), "status reset");
    NA_CUDA(cudaMemsetAsync(dev + kLevelsOff, 0, kLevelSlots * sizeof(LevelSlot), s), "level reset");
    if (!pj.blob.empty())
      NA_CUDA(cudaMemcpyAsync(dev + kBlobOff, pj.blob.data(), pj.blob.size(), cudaMemcpyHostToDevice, s),
              "blob upload");
    if (n_tiles)
      NA_CUDA(cudaMemcpyAsync(dev + kTilesOff, tiles.data(), n_tiles * sizeof(Tile), cudaMemcpyHostToDevice, s),
              "tile upload");
    // Once the kernel is launched it uses the shared array until it ends: every return from here on
    // first waits for the stream, so that the next pass or call never resets the array under it.
    struct StreamGuard {
      cudaStream_t s;
      bool armed = false;
      ~StreamGuard() {
        if (armed) cudaStreamSynchronize(s);
      }
    } guard{s};
    if (n_tiles) {
      const size_t grid = std::max<size_t>(1, std::min<size_t>(n_tiles, static_cast<size_t>(per_sm) * sms));
      kernel<<<static_cast<uint32_t>(grid), kBlock, d.smem_bytes, s>>>(
          reinterpret_cast<const JobDesc*>(dev + kDescOff), reinterpret_cast<const Tile*>(dev + kTilesOff),
          static_cast<uint32_t>(n_tiles), reinterpret_cast<QueueCtl*>(dev + kQueueOff), nullptr,
          reinterpret_cast<unsigned long long*>(dev + kStatusOff), nullptr);
      guard.armed = true;
      NA_CUDA(cudaGetLastError(), "engine launch failed");
    }
    unsigned long long status = 0;
    NA_CUDA(cudaMemcpyAsync(lv, dev + kLevelsOff, sizeof(lv), cudaMemcpyDeviceToHost, s), "level download");
    NA_CUDA(cudaMemcpyAsync(cnt, dev + kCountersOff, sizeof(cnt), cudaMemcpyDeviceToHost, s), "counter download");
    NA_CUDA(cudaMemcpyAsync(&status, dev + kStatusOff, 8, cudaMemcpyDeviceToHost, s), "status download");
    NA_CUDA(cudaStreamSynchronize(s), "engine run failed");
    guard.armed = false;
    if (status == kErrStageTimeout) NA_FAIL(SQSG_ERR_TIMEOUT, "shared-memory staging wait timed out on the device");
    if (status) NA_FAIL(SQSG_ERR_CUDA, "device error");
    const sqsg_status cs = guarded([&] { check_job_counters(cnt); });
    if (cs != SQSG_OK) {
      char msg[512];
      sqsg_last_error(msg, sizeof(msg));
      NA_FAIL(cs, msg);
    }
    return ok();
  };
  const auto t0 = std::chrono::steady_clock::now();
  // While the search threshold is still high the table takes every new objective, and it overflows
  // when a job has more distinct objectives than slots before the warps' best lists fill (keep+1
  // distinct values per warp). Every pass evaluates the same configurations, so a pass that starts
  // from a threshold at or above the (keep+1)-th best distinct objective yields the exact levels. Two
  // such bounds come out of an overflowed pass: the final device threshold, and the (keep+1)-th
  // smallest key the table did take (those keys are objectives of the job). The next pass starts
  // from the smaller one; each pass keeps about (keep+1)/kLevelSlots of the objectives below the
  // previous bound, so a few passes suffice.
  constexpr int kMaxPasses = 8;
  unsigned long long threshold = ord_bits(maxv);
  for (int p = 0;; ++p) {
    NA_TRY(pass(threshold));
    if (!cnt[kLevelOverflow]) break;
    if (p + 1 == kMaxPasses) break;  // reported as an overflow below
    static unsigned long long keys[kLevelSlots];
    uint32_t nk = 0;
    for (int k = 0; k < kLevelSlots; ++k)
      if (lv[k].key) keys[nk++] = lv[k].key;
    unsigned long long next = cnt[kThreshold];
    if (nk > job.keep) {
      std::nth_element(keys, keys + job.keep, keys + nk);
      next = std::min(next, keys[job.keep]);
    }
    if (next >= threshold) break;  // no tighter bound: reported as an overflow below
    threshold = next;
  }
  const auto t1 = std::chrono::steady_clock::now();
  // the keep+1 smallest objective keys, by insertion into a fixed array (guarded by g_mutex)
  const uint32_t want = static_cast<uint32_t>(job.keep + 1);
  static LevelSlot best[kMaxKeep + 1];
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
    stats->best_rank = ~0ull;  // not reported: this entry point keeps no configuration records
    stats->best_objective = nb ? from_ord(best[0].key) : std::numeric_limits<double>::infinity();
    const uint64_t ns = static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count());
    stats->timings_ns[SQSG_TIMING_TOTAL] = ns;
    stats->timings_ns[SQSG_TIMING_LOOP] = ns;
  }
  if (cnt[kLevelOverflow]) NA_FAIL(SQSG_ERR_CAPACITY, "the objective-level table overflowed; levels are incomplete");
  if (nb > cap) NA_FAIL(SQSG_ERR_CAPACITY, "level capacity too small");
  return ok();
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
  return report(e.status, e.msg.c_str());
}

}  // extern "C"
