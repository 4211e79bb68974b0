// Peak-rate microbenchmarks for the roofline of the SQS engine, whose bound is on-chip (shared-memory
// loads and 32-bit integer issue), not HBM or tensor cores. Each kernel saturates one resource on
// every SM and reports the achieved rate; the benchmark divides the engine's algorithmic work by it.

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "sqsg_internal.h"

namespace sqsg {

constexpr int kMbBlock = 256;
constexpr int kMbIters = 4096;

// Conflict-free 32-bit shared-memory loads: every warp reads 32 consecutive words per instruction,
// eight independent chains per thread.
__global__ void __launch_bounds__(kMbBlock) mb_smem_kernel(unsigned* out, unsigned seed) {
  __shared__ unsigned buf[kMbBlock * 8];
  for (int i = threadIdx.x; i < kMbBlock * 8; i += kMbBlock) buf[i] = seed ^ (i * 2654435761u);
  __syncthreads();
  unsigned acc[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc[k] = 0;
  unsigned idx = threadIdx.x;
  for (int it = 0; it < kMbIters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] ^= buf[(idx + k * kMbBlock) & (kMbBlock * 8 - 1)];
    idx = (idx + 32) & (kMbBlock * 8 - 1);
  }
  unsigned r = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) r ^= acc[k];
  if (r == 0x9e3779b9u) out[0] = r;  // keeps the loads alive
}

// Independent 32-bit integer add/xor chains (IADD3 / LOP3 class), eight per thread.
__global__ void __launch_bounds__(kMbBlock) mb_int_kernel(unsigned* out, unsigned seed) {
  unsigned a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 7u + k;
  for (int it = 0; it < kMbIters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      a[k] = a[k] + (a[k] ^ 0x5bd1e995u);
      a[k] = a[k] ^ (a[k] + 0x27d4eb2du);
    }
  }
  unsigned r = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) r ^= a[k];
  if (r == 0x9e3779b9u) out[0] = r;
}

// Independent population-count chains, eight per thread: per step one logic op, one POPC and one add
// (the lattice path's AND-popcount-accumulate).
__global__ void __launch_bounds__(kMbBlock) mb_popc_kernel(unsigned* out, unsigned seed) {
  unsigned a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 7u + k;
  const unsigned m = seed * 0x9e3779b9u;
  for (int it = 0; it < kMbIters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] += static_cast<unsigned>(__popc(a[k] ^ m));
  }
  unsigned r = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) r ^= a[k];
  if (r == 0x9e3779b9u) out[0] = r;
}

}  // namespace sqsg

using namespace sqsg;

extern "C" {

// kind 0: shared-memory load bandwidth in bytes/s; kind 1: 32-bit integer ops/s (lane operations);
// kind 2: 32-bit population counts per second (with a logic op and an add each).
// Also returns the kernel time in seconds.
sqsg_status sqsg_microbench(int kind, int device, double* rate, double* seconds) {
  return guarded([&] {
    if (!rate) throw std::invalid_argument("null pointer");
    if (kind < 0 || kind > 2) throw std::invalid_argument("microbenchmark kind must be 0, 1 or 2");
    if (cudaSetDevice(device) != cudaSuccess) throw cuda_error("cudaSetDevice failed");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    unsigned* out = nullptr;
    if (cudaMalloc(&out, 16) != cudaSuccess) throw cuda_error("cudaMalloc failed");
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int grid = sms * 8;
    double best = 0, best_t = 0;
    for (int rep = 0; rep < 4; ++rep) {
      cudaEventRecord(a);
      if (kind == 0)
        mb_smem_kernel<<<grid, kMbBlock>>>(out, 1u + rep);
      else if (kind == 1)
        mb_int_kernel<<<grid, kMbBlock>>>(out, 1u + rep);
      else
        mb_popc_kernel<<<grid, kMbBlock>>>(out, 1u + rep);
      cudaEventRecord(b);
      cudaEventSynchronize(b);
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      const double threads = static_cast<double>(grid) * kMbBlock;
      // bytes (kind 0: 8 loads of 4 bytes), lane ops (kind 1: 4 per chain step), popcounts (kind 2)
      const double work = threads * kMbIters * 8 * (kind == 2 ? 1.0 : 4.0);
      const double r = work / (ms * 1e-3);
      if (rep > 0 && r > best) {
        best = r;
        best_t = ms * 1e-3;
      }
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    if (e != cudaSuccess) throw cuda_error(cudaGetErrorString(e));
    *rate = best;
    if (seconds) *seconds = best_t;
  });
}

}  // extern "C"
