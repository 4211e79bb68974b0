// sqsg_engine_lat5: the lattice path for parts of at most five species (up to 10 species-pair counters
// and the planes of 4 species per lane), 3 CTAs per SM.
#include "engine_device.cuh"
#include "kernels.h"

namespace sqsg {

__global__ void __launch_bounds__(kBlock, kMinBlocksLat5)
    sqsg_engine_lat5(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                     const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done) {
  engine_body<false, false, 5>(jobs, tiles, n_tiles, q, cancel, status, done);
}

}  // namespace sqsg
