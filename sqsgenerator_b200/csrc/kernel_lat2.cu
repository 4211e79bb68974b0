// sqsg_engine_lat2: the lattice path for binary parts (one species-pair counter and one plane per
// unit-cell site and lane), 4 CTAs per SM.
#include "engine_device.cuh"
#include "kernels.h"

namespace sqsg {

__global__ void __launch_bounds__(kBlock, kMinBlocksLat2)
    sqsg_engine_lat2(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                     const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done) {
  engine_body<false, false, 2>(jobs, tiles, n_tiles, q, cancel, status, done);
}

}  // namespace sqsg
