// sqsg_materialize: full records for selected candidates.
//
// The engine appends only (objective, id) per candidate. A configuration depends on nothing but the
// job and its id — random mode: the shuffle (shuffle_part) of the staged initial arrangement with the
// words seeded by id; systematic mode: the multiset permutation of rank id (core/permutation.h:52-78) — so
// the full record of a selected candidate (species, per-part objective and SRO cube) is rebuilt here,
// once, through the general pair-stream path: ordered bonds (core/optimization.h:74-77), objective and
// SRO (optimization.h:79-103), parts summed left to right (sqs.h:417-418). In the reference-stream
// debug mode a configuration is rebuilt by replaying its block's chain up to its id. The rebuilt objective must
// equal the candidate's bit for bit; every mismatch is counted in *bad (the host raises an error).
#include "engine_device.cuh"
#include "kernels.h"

namespace sqsg {

template <class T, int KW, bool SYS>
__device__ __forceinline__ void materialize_one(const JobDesc& J, uint8_t* smem, const Cand& c, uint8_t* rec, int t,
                                                unsigned long long* bad) {
  using F = FP<T>;
  const uint64_t id = c.id;
  for (uint32_t p = 0; p < J.n_parts; ++p) init_column(smem, J.parts[p], t);
  if (SYS) {
    const PartDesc& P = J.parts[0];
    const uint32_t* win = reinterpret_cast<const uint32_t*>(part_base(smem, P) + P.win_off);
    unrank_window(part_base(smem, P) + P.col_off + 4 * t, P, win[0], win[1] - win[0], id, J.total);
  } else if (J.chain) {
    // reference-stream mode: replay the configuration's block from its start (run_tile_chain)
    const uint64_t first = chain_block_start(J, chain_block_of(J, id));
    for (uint32_t p = 0; p < J.n_parts; ++p) {
      unsigned long long st = chain_state(J, J.parts[p], first);
      const uint64_t shuffles = id - first + (J.chain_split ? 1 : 0);
      for (uint64_t k = 0; k < shuffles; ++k) shuffle_part_rapid(smem, J.parts[p], t, st);
    }
  } else {
    const uint32_t k0 = static_cast<uint32_t>(J.seed), k1 = static_cast<uint32_t>(J.seed >> 32);
    for (uint32_t p = 0; p < J.n_parts; ++p) shuffle_part(smem, J.parts[p], t, 0u, id, p, k0, k1);
  }
  T total = T(0);
  for (uint32_t p = 0; p < J.n_parts; ++p) {
    const PartDesc& P = J.parts[p];
    count_part<KW>(smem, J.blob, P, t);
    const T o = objective_part<T>(smem, P, t, reinterpret_cast<T*>(rec + P.rec_sro_off));
    *reinterpret_cast<T*>(rec + P.rec_obj_off) = o;
    const uint8_t* col = part_base(smem, P) + P.col_off + 4 * t;
    for (uint32_t x = 0; x < P.n_sites; ++x) rec[P.rec_species_off + x] = col[site_off(x)] >> 3;
    total = p == 0 ? o : F::add(total, o);
  }
  *reinterpret_cast<T*>(rec) = total;
  *reinterpret_cast<uint64_t*>(rec + 8) = id;
  if (static_cast<double>(total) != c.objective) atomicAdd(bad, 1ull);
}

template <bool SYS>
__device__ __forceinline__ void materialize_dispatch(const JobDesc& J, uint8_t* smem, const Cand& c, uint8_t* rec,
                                                     int t, unsigned long long* bad) {
  if (J.prec == 1) {
    if (J.kw == 1)
      materialize_one<double, 1, SYS>(J, smem, c, rec, t, bad);
    else
      materialize_one<double, 2, SYS>(J, smem, c, rec, t, bad);
  } else {
    if (J.kw == 1)
      materialize_one<float, 1, SYS>(J, smem, c, rec, t, bad);
    else
      materialize_one<float, 2, SYS>(J, smem, c, rec, t, bad);
  }
}

__global__ void __launch_bounds__(kBlock)
    sqsg_materialize(const JobDesc* __restrict__ job, const Cand* __restrict__ cands, uint32_t n,
                     uint8_t* __restrict__ out, unsigned long long* bad) {
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ JobDesc sj;
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(job);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&sj);
    for (uint32_t i = threadIdx.x; i < sizeof(JobDesc) / 4; i += kBlock) dst[i] = src[i];
  }
  __syncthreads();
  // staged sections with plain loads (a selection launches this kernel once)
  for (uint32_t p = 0; p < sj.n_parts; ++p) {
    const uint4* src = reinterpret_cast<const uint4*>(sj.blob + sj.parts[p].blob_off);
    uint4* dst = reinterpret_cast<uint4*>(smem + sj.parts[p].smem_off);
    for (uint32_t i = threadIdx.x; i < sj.parts[p].static_bytes / 16; i += kBlock) dst[i] = src[i];
  }
  __syncthreads();
  const uint32_t k = blockIdx.x * kBlock + threadIdx.x;
  if (k >= n) return;
  uint8_t* rec = out + static_cast<size_t>(k) * sj.record_bytes;
  if (sj.mode == 1)
    materialize_dispatch<true>(sj, smem, cands[k], rec, threadIdx.x, bad);
  else
    materialize_dispatch<false>(sj, smem, cands[k], rec, threadIdx.x, bad);
}

}  // namespace sqsg
