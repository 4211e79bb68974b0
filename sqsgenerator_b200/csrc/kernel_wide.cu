// sqsg_engine_wide: the persistent engine holding the general pair-stream path at 128 registers (its
// pair loop spills at 96, and its shared memory allows at most 4 CTAs per SM anyway).
#include "engine_device.cuh"
#include "kernels.h"

namespace sqsg {

__global__ void __launch_bounds__(kBlock, kMinBlocksWide)
    sqsg_engine_wide(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                     const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done) {
  engine_body<true, false, 0>(jobs, tiles, n_tiles, q, cancel, status, done);
}

}  // namespace sqsg
