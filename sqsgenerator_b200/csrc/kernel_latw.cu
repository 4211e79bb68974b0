// sqsg_engine_latw: the lattice path for supercells of 65 to 128 unit cells (cell sets of two 64-bit
// words) and parts of at most five species, 2 CTAs per SM.
#include "engine_device.cuh"
#include "kernels.h"

namespace sqsg {

__global__ void __launch_bounds__(kBlock, kMinBlocksLatW)
    sqsg_engine_latw(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                     const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done) {
  engine_body<false, false, 5, 2>(jobs, tiles, n_tiles, q, cancel, status, done);
}

}  // namespace sqsg
