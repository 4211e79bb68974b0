// sqsg_engine_lat: the persistent engine holding the lattice path (bonds from translated bit planes of
// a supercell, see run_tile_lat) for parts of up to eight species. Its per-lane state for eight
// species (28 species-pair counters, translated and current planes of 7 species) needs more than 128
// registers, so the kernel allows 2 CTAs per SM at up to 255 registers instead of spilling. Jobs of
// two species or at most five run in sqsg_engine_lat2 / sqsg_engine_lat5, whose smaller state leaves
// room for more CTAs per SM.
#include "engine_device.cuh"
#include "kernels.h"

namespace sqsg {

__global__ void __launch_bounds__(kBlock, kMinBlocksLat)
    sqsg_engine_lat(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                    const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done) {
  engine_body<false, false, 8>(jobs, tiles, n_tiles, q, cancel, status, done);
}

}  // namespace sqsg
