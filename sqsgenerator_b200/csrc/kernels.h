// Declarations of the engine kernels (each defined in its own translation unit, so that they compile
// in parallel): host code launches them through these.
#pragma once

#include <cstdint>

#include "engine.cuh"

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

// sqsg_engine_lat — the lattice path (supercells whose pairs are whole translation classes).
__global__ void __launch_bounds__(kBlock, kMinBlocksLat)
    sqsg_engine_lat(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                    const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done);

// Rebuilds the full records (selection order) of n candidates of one job; counts objective mismatches.
__global__ void __launch_bounds__(kBlock)
    sqsg_materialize(const JobDesc* __restrict__ job, const Cand* __restrict__ cands, uint32_t n,
                     uint8_t* __restrict__ out, unsigned long long* bad);

}  // namespace sqsg
