// Declarations of the engine kernels (each defined in its own translation unit, so that they compile
// in parallel): host code launches them through these.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>

#include "engine.cuh"
#include "sqsg_internal.h"

namespace sqsg {

// The persistent tile kernel compiled two ways (see engine_device.cuh, engine_body):
//  sqsg_engine_mask — the binary bit-mask path alone, 96 registers (5 CTAs per SM);
//  sqsg_engine_wide — the general pair-stream path alone, 128 registers (no spills in the pair loop);
//                     a bit-mask job given to it runs the general path, which holds all its data too.
__global__ void __launch_bounds__(kBlock, kMinBlocks)
    sqsg_engine_mask(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                     const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done);

__global__ void __launch_bounds__(kBlock, kMinBlocksWide)
    sqsg_engine_wide(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                     const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done);

// The lattice path (supercells whose pairs are whole translation classes), by the largest species
// count of a job's parts: sqsg_engine_lat2 (binary, 4 CTAs per SM), sqsg_engine_lat5 (at most five,
// 3 CTAs per SM) and sqsg_engine_lat (at most eight, 2 CTAs per SM).
__global__ void __launch_bounds__(kBlock, kMinBlocksLat)
    sqsg_engine_lat(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                    const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done);
__global__ void __launch_bounds__(kBlock, kMinBlocksLat2)
    sqsg_engine_lat2(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                     const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done);
__global__ void __launch_bounds__(kBlock, kMinBlocksLat5)
    sqsg_engine_lat5(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                     const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done);
// sqsg_engine_latw: lattice jobs of 65 to 128 unit cells (two-word cell sets), at most five species.
__global__ void __launch_bounds__(kBlock, kMinBlocksLatW)
    sqsg_engine_latw(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                     const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done);

// Rebuilds the full records (selection order) of n candidates of one job; counts objective mismatches.
__global__ void __launch_bounds__(kBlock)
    sqsg_materialize(const JobDesc* __restrict__ job, const Cand* __restrict__ cands, uint32_t n,
                     uint8_t* __restrict__ out, unsigned long long* bad);

using EngineKernel = void (*)(const JobDesc*, const Tile*, uint32_t, QueueCtl*, const volatile int32_t*,
                              unsigned long long*, volatile uint32_t*);

// Kernel kinds: each job runs in the kernel that holds its path. A bit-mask job (k2) runs in
// sqsg_engine_mask; a lattice job of up to 64 cells in the lattice kernel of its largest species count
// (lat_kmax 2, at most 5, at most 8), one of 65-128 cells in sqsg_engine_latw; every other job in
// sqsg_engine_wide (which may also take bit-mask jobs: their columns and pair stream exist too;
// sqsg_engine_lat likewise takes every lattice job of up to 64 cells). A job given to a kernel without
// its path is skipped on the device and flagged kErrBadJob in its counters.
enum KernelKind : int {
  kKindMask = 0, kKindWide = 1, kKindLat = 2, kKindLat2 = 3, kKindLat5 = 4, kKindLatW = 5, kKindCount = 6
};
inline bool is_lattice_kind(int kind) { return kind >= kKindLat && kind <= kKindLatW; }
inline int kind_of(const JobDesc& d) {
  if (d.k2) return kKindMask;
  if (!d.lat) return kKindWide;
  if (d.lat_words == 2) return kKindLatW;
  return d.lat_kmax <= 2 ? kKindLat2 : (d.lat_kmax <= 5 ? kKindLat5 : kKindLat);
}
inline EngineKernel kernel_of(int kind) {
  switch (kind) {
    case kKindMask: return sqsg_engine_mask;
    case kKindLat: return sqsg_engine_lat;
    case kKindLat2: return sqsg_engine_lat2;
    case kKindLat5: return sqsg_engine_lat5;
    case kKindLatW: return sqsg_engine_latw;
    default: return sqsg_engine_wide;
  }
}
inline const char* kernel_name(int kind) {
  switch (kind) {
    case kKindMask: return "sqsg_engine_mask";
    case kKindLat: return "sqsg_engine_lat";
    case kKindLat2: return "sqsg_engine_lat2";
    case kKindLat5: return "sqsg_engine_lat5";
    case kKindLatW: return "sqsg_engine_latw";
    default: return "sqsg_engine_wide";
  }
}

// Throws for the device-side errors a job's counters carry: a staging timeout, a job launched in a
// kernel without its path, and lattice objectives that differ from the pair-stream path's (traces).
inline void check_job_counters(const unsigned long long* cnt) {
  if (cnt[kError] == kErrStageTimeout) throw timeout_error("shared-memory staging wait timed out on the device");
  if (cnt[kError] == kErrBadJob) throw std::logic_error("internal error: a job was launched in a kernel without its path");
  if (cnt[kError]) throw cuda_error("device error code " + std::to_string(cnt[kError]));
  if (cnt[kMismatch])
    throw cuda_error("internal error: " + std::to_string(cnt[kMismatch]) +
                     " lattice-path objectives differ from the pair-stream path's");
}

}  // namespace sqsg
