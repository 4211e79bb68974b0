// sqsg_engine_mask: the persistent engine holding the binary bit-mask path only. Without the general
// path's code nothing forces spills at 96 registers (5 CTAs per SM).
#include "engine_device.cuh"
#include "kernels.h"

namespace sqsg {

__global__ void __launch_bounds__(kBlock, kMinBlocks)
    sqsg_engine_mask(const JobDesc* __restrict__ jobs, const Tile* __restrict__ tiles, uint32_t n_tiles, QueueCtl* q,
                     const volatile int32_t* cancel, unsigned long long* status, volatile uint32_t* done) {
  engine_body<false, true, 0>(jobs, tiles, n_tiles, q, cancel, status, done);
}

}  // namespace sqsg
