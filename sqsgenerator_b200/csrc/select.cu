// Result-set selection on the device (see select.h). The reference keeps, per exact objective, a set
// of distinct configurations (include/sqsgen/core/results.h:42-99) and returns the objectives in
// ascending order; the engine's candidate buffer holds every evaluation at or below the final
// (keep+1)-th best distinct objective, in no particular order and with repeats in random mode.
//
// Steps, all on one stream:
//   1. keep the records whose objective is one of the exact level values (the keep+1 smallest);
//   2. radix-sort them by (level index, id) in one 64-bit key;
//   3. random mode: sort the positions by a 64-bit hash of the species and mark every record whose
//      species equal those of an earlier record (same level, smaller id) in its hash run;
//   4. cap each objective at max_per_objective+1 records (the reference's `>` test);
//   5. gather objective, sub-objectives, species, SRO and id into dense arrays and copy them out.

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>

#include "host_copy.h"
#include "kernels.h"
#include "select.h"
#include "sqsg_internal.h"

namespace sqsg {

#define SEL_CHECK(expr)                                                                               \
  do {                                                                                                \
    cudaError_t err__ = (expr);                                                                       \
    if (err__ != cudaSuccess)                                                                         \
      throw cuda_error(std::string(#expr) + ": " + cudaGetErrorString(err__));                       \
  } while (0)

// Stream-ordered allocations: growing a buffer never waits for other streams' kernels (a plain
// cudaFree would wait for the whole device, including persistent kernels of other jobs).
void SelectScratch::release() {
  for (int k = 0; k < kSlots; ++k) {
    if (buf[k]) cudaFreeAsync(buf[k], stream);
    buf[k] = nullptr;
    size[k] = 0;
  }
  if (stream) cudaStreamSynchronize(stream);
  stream = nullptr;
  for (int k = 0; k < 2; ++k) {
    if (bounce[k]) cudaFreeHost(bounce[k]);
    if (bounce_done[k]) cudaEventDestroy(bounce_done[k]);
    bounce[k] = nullptr;
    bounce_done[k] = nullptr;
  }
}

namespace {

constexpr size_t kBounceBytes = 32u << 20;

// Device-to-host copy into pageable memory. Large copies go through two pinned buffers: the copy
// engine fills one while the host drains the other (several times the driver's pageable rate).
void copy_out(SelectScratch& S, cudaStream_t st, void* dst, const void* src, size_t bytes) {
  if (bytes < (64u << 10)) {
    SEL_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    return;
  }
  for (int k = 0; k < 2; ++k) {
    if (!S.bounce[k]) SEL_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&S.bounce[k]), kBounceBytes, cudaHostAllocDefault));
    if (!S.bounce_done[k]) SEL_CHECK(cudaEventCreateWithFlags(&S.bounce_done[k], cudaEventDisableTiming));
  }
  size_t pend_off[2] = {}, pend_len[2] = {};
  bool pend[2] = {false, false};
  int b = 0;
  auto drain = [&](int k) {
    SEL_CHECK(cudaEventSynchronize(S.bounce_done[k]));
    parallel_copy(static_cast<uint8_t*>(dst) + pend_off[k], S.bounce[k], pend_len[k]);
    pend[k] = false;
  };
  for (size_t off = 0; off < bytes; off += kBounceBytes, b ^= 1) {
    const size_t len = std::min(kBounceBytes, bytes - off);
    if (pend[b]) drain(b);
    SEL_CHECK(cudaMemcpyAsync(S.bounce[b], static_cast<const uint8_t*>(src) + off, len, cudaMemcpyDeviceToHost, st));
    SEL_CHECK(cudaEventRecord(S.bounce_done[b], st));
    pend[b] = true;
    pend_off[b] = off;
    pend_len[b] = len;
  }
  for (int k = 0; k < 2; ++k)
    if (pend[(b + k) % 2]) drain((b + k) % 2);
}

}  // namespace

// The device's default pool keeps what select_on_device frees, so later calls reuse it.
static void keep_pool_memory() {
  static std::atomic<uint64_t> done_mask{0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev >= 64) return;
  if (done_mask.load() & (1ull << dev)) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done_mask.fetch_or(1ull << dev);
}

void* SelectScratch::get(int slot, size_t bytes) {
  bytes = std::max<size_t>(bytes, 256);
  if (size[slot] < bytes) {
    keep_pool_memory();
    if (buf[slot]) SEL_CHECK(cudaFreeAsync(buf[slot], stream));
    buf[slot] = nullptr;
    size[slot] = 0;
    SEL_CHECK(cudaMallocAsync(&buf[slot], bytes, stream));
    size[slot] = bytes;
  }
  return buf[slot];
}

namespace {

// Level keys (ord_bits of the keep+1 smallest distinct objectives, ascending) in device memory.
__device__ __forceinline__ int level_of(const unsigned long long* __restrict__ L, uint32_t nl, unsigned long long key) {
  int lo = 0, hi = static_cast<int>(nl) - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const unsigned long long k = L[mid];
    if (k == key) return mid;
    if (k < key)
      lo = mid + 1;
    else
      hi = mid - 1;
  }
  return -1;
}

__global__ void k_flag_levels(const Cand* __restrict__ c, uint32_t n, const unsigned long long* __restrict__ L,
                              uint32_t nl, uint8_t* __restrict__ flag, uint32_t* __restrict__ iota) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  flag[i] = level_of(L, nl, ord_bits(c[i].objective)) >= 0 ? 1 : 0;
  iota[i] = i;
}

__global__ void k_keys(const Cand* __restrict__ c, const uint32_t* __restrict__ sel, uint32_t m,
                       const unsigned long long* __restrict__ L, uint32_t nl, uint32_t id_bits,
                       unsigned long long* __restrict__ key, uint32_t* __restrict__ pos) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const Cand x = c[sel[j]];
  key[j] = (static_cast<unsigned long long>(level_of(L, nl, ord_bits(x.objective))) << id_bits) | x.id;
  pos[j] = j;
}

// out[k] = candidate of sorted position order[k]
__global__ void k_gather_cands(const Cand* __restrict__ c, const uint32_t* __restrict__ sel,
                               const uint32_t* __restrict__ pos_s, const uint32_t* __restrict__ order, uint32_t m,
                               Cand* __restrict__ out) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  out[k] = c[sel[pos_s[order ? order[k] : k]]];
}

__global__ void k_hash(const uint8_t* __restrict__ recs, RecordLayout lay, uint32_t m, unsigned long long* __restrict__ hash,
                       uint32_t* __restrict__ iota) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const uint8_t* r = recs + static_cast<size_t>(j) * lay.record_bytes;
  unsigned long long h = 0xcbf29ce484222325ull;  // FNV-1a over the species bytes of all parts
  for (uint32_t p = 0; p < lay.n_parts; ++p)
    for (uint32_t x = 0; x < lay.n_sites[p]; ++x) h = (h ^ r[lay.species_off[p] + x]) * 0x100000001b3ull;
  hash[j] = h;
  iota[j] = j;
}

__device__ __forceinline__ bool same_species(const uint8_t* a, const uint8_t* b, const RecordLayout& lay) {
  for (uint32_t p = 0; p < lay.n_parts; ++p)
    for (uint32_t x = 0; x < lay.n_sites[p]; ++x)
      if (a[lay.species_off[p] + x] != b[lay.species_off[p] + x]) return false;
  return true;
}

// Records are in (level, id) order; r runs over the (hash, position) order and q[r] is the record.
// A record is a repeat when an earlier record of its hash run has the same level and the same species
// (an earlier position in (level, id) order: the smallest id stays).
__global__ void k_mark_repeats(const uint8_t* __restrict__ recs, RecordLayout lay,
                               const unsigned long long* __restrict__ key_s, const unsigned long long* __restrict__ hs,
                               const uint32_t* __restrict__ q, uint32_t m, uint32_t id_bits, uint8_t* __restrict__ keep) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const uint32_t p = q[r];
  const unsigned long long lev = key_s[p] >> id_bits;
  const uint8_t* a = recs + static_cast<size_t>(p) * lay.record_bytes;
  bool repeat = false;
  for (uint32_t r2 = r; r2 > 0 && hs[r2 - 1] == hs[r]; --r2) {
    const uint32_t p2 = q[r2 - 1];
    if ((key_s[p2] >> id_bits) != lev) continue;
    if (same_species(recs + static_cast<size_t>(p2) * lay.record_bytes, a, lay)) {
      repeat = true;
      break;
    }
  }
  keep[p] = repeat ? 0 : 1;
}

__global__ void k_iota(uint32_t m, uint32_t* __restrict__ iota) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) iota[i] = i;
}

// kp: kept positions in (level, id) order. start[level] = index in kp of the level's first record.
__global__ void k_level_starts(const uint32_t* __restrict__ kp, const unsigned long long* __restrict__ key_s,
                               uint32_t m, uint32_t id_bits, uint32_t* __restrict__ start) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  const uint32_t lev = static_cast<uint32_t>(key_s[kp[t]] >> id_bits);
  if (t == 0 || static_cast<uint32_t>(key_s[kp[t - 1]] >> id_bits) != lev) start[lev] = t;
}

__global__ void k_cap(const uint32_t* __restrict__ kp, const unsigned long long* __restrict__ key_s, uint32_t m,
                      uint32_t id_bits, const uint32_t* __restrict__ start, unsigned long long cap,
                      uint8_t* __restrict__ flag) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  const uint32_t lev = static_cast<uint32_t>(key_s[kp[t]] >> id_bits);
  flag[t] = static_cast<unsigned long long>(t - start[lev]) <= cap ? 1 : 0;
}

struct OutLayout {
  uint8_t* objective;
  uint8_t* sub_objective;
  uint8_t* species;
  uint8_t* sro;
  unsigned long long* id;
  uint32_t species_total, sro_total;
  uint32_t species_prefix[kMaxParts], sro_prefix[kMaxParts];
};

// One warp per selected record: record order[t] (or t) into dense output row t.
__global__ void k_gather(const uint8_t* __restrict__ recs, RecordLayout lay, const uint32_t* __restrict__ order,
                         uint32_t m, OutLayout o) {
  const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (t >= m) return;
  const uint8_t* r = recs + static_cast<size_t>(order ? order[t] : t) * lay.record_bytes;
  const uint32_t tsz = lay.tsz;
  if (lane < tsz) o.objective[static_cast<size_t>(t) * tsz + lane] = r[lane];
  if (lane < 8) reinterpret_cast<uint8_t*>(o.id)[static_cast<size_t>(t) * 8 + lane] = r[8 + lane];
  for (uint32_t p = 0; p < lay.n_parts; ++p) {
    if (lane < tsz) o.sub_objective[(static_cast<size_t>(t) * lay.n_parts + p) * tsz + lane] = r[lay.obj_off[p] + lane];
    uint8_t* sp = o.species + static_cast<size_t>(t) * o.species_total + o.species_prefix[p];
    for (uint32_t x = lane; x < lay.n_sites[p]; x += 32) sp[x] = r[lay.species_off[p] + x];
    uint8_t* sr = o.sro + static_cast<size_t>(t) * o.sro_total + o.sro_prefix[p];
    for (uint32_t x = lane; x < lay.sro_bytes[p]; x += 32) sr[x] = r[lay.sro_off[p] + x];
  }
}

inline uint32_t blocks(uint64_t n, uint32_t per) { return static_cast<uint32_t>((n + per - 1) / per); }

template <class Fn> size_t cub_bytes(Fn&& fn) {
  size_t b = 0;
  SEL_CHECK(fn(nullptr, b));
  return b;
}

uint32_t select_flagged(SelectScratch& S, cudaStream_t st, const uint32_t* in, const uint8_t* flag, uint32_t* out,
                        uint32_t n) {
  auto* d_num = static_cast<uint32_t*>(S.get(9, 256));
  const size_t tb = cub_bytes([&](void* p, size_t& b) {
    return cub::DeviceSelect::Flagged(p, b, in, flag, out, d_num, n, st);
  });
  void* tmp = S.get(8, tb);
  size_t b = tb;
  SEL_CHECK(cub::DeviceSelect::Flagged(tmp, b, in, flag, out, d_num, n, st));
  uint32_t m = 0;
  SEL_CHECK(cudaMemcpyAsync(&m, d_num, sizeof(m), cudaMemcpyDeviceToHost, st));
  SEL_CHECK(cudaStreamSynchronize(st));
  return m;
}

template <class K, class V>
void sort_pairs(SelectScratch& S, cudaStream_t st, const K* kin, K* kout, const V* vin, V* vout, uint32_t n,
                int end_bit) {
  const size_t tb = cub_bytes([&](void* p, size_t& b) {
    return cub::DeviceRadixSort::SortPairs(p, b, kin, kout, vin, vout, n, 0, end_bit, st);
  });
  void* tmp = S.get(8, tb);
  size_t b = tb;
  SEL_CHECK(cub::DeviceRadixSort::SortPairs(tmp, b, kin, kout, vin, vout, n, 0, end_bit, st));
}

// Per-level cap on positions kp (m entries, (level, id) order): returns the kept count, into out.
uint32_t cap_levels(SelectScratch& S, cudaStream_t st, const uint32_t* kp, const unsigned long long* key_s, uint32_t m,
                    uint32_t id_bits, uint32_t n_levels, int64_t cap, uint32_t* out) {
  auto* start = static_cast<uint32_t*>(S.get(13, size_t(n_levels) * 4));
  auto* cflag = static_cast<uint8_t*>(S.get(11, m));
  SEL_CHECK(cudaMemsetAsync(start, 0, size_t(n_levels) * 4, st));
  k_level_starts<<<blocks(m, 256), 256, 0, st>>>(kp, key_s, m, id_bits, start);
  SEL_CHECK(cudaGetLastError());
  k_cap<<<blocks(m, 256), 256, 0, st>>>(kp, key_s, m, id_bits, start, static_cast<unsigned long long>(cap), cflag);
  SEL_CHECK(cudaGetLastError());
  return select_flagged(S, st, kp, cflag, out, m);
}

}  // namespace

uint64_t materialize(SelectScratch& S, cudaStream_t st, const Materializer& mat, const Cand* d_cands, uint32_t m,
                     uint8_t* d_out) {
  if (S.stream != st) {
    S.release();
    S.stream = st;
  }
  if (m == 0) return 0;
  auto* d_job = static_cast<JobDesc*>(S.get(16, sizeof(JobDesc)));
  auto* d_bad = static_cast<unsigned long long*>(S.get(17, 256));
  SEL_CHECK(cudaMemcpyAsync(d_job, &mat.job, sizeof(JobDesc), cudaMemcpyHostToDevice, st));
  SEL_CHECK(cudaMemsetAsync(d_bad, 0, 8, st));
  const int err = raise_dynamic_smem(reinterpret_cast<const void*>(sqsg_materialize), mat.smem);
  if (err != 0) throw cuda_error(std::string("cudaFuncSetAttribute(sqsg_materialize): ") +
                                 cudaGetErrorString(static_cast<cudaError_t>(err)));
  sqsg_materialize<<<blocks(m, kBlock), kBlock, mat.smem, st>>>(d_job, d_cands, m, d_out, d_bad);
  SEL_CHECK(cudaGetLastError());
  unsigned long long bad = 0;
  SEL_CHECK(cudaMemcpyAsync(&bad, d_bad, 8, cudaMemcpyDeviceToHost, st));
  SEL_CHECK(cudaStreamSynchronize(st));
  return bad;
}

namespace {

__global__ void k_compact_dedup(const DedupSlot* __restrict__ tab, uint64_t slots, Cand* __restrict__ out, uint64_t cap,
                                unsigned long long* __restrict__ count) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < slots;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const DedupSlot e = tab[i];
    if (e.key == kDedupEmpty) continue;
    const unsigned long long k = atomicAdd(count, 1ull);
    if (k < cap) out[k] = Cand{e.objective, e.id};
  }
}

}  // namespace

uint64_t compact_dedup(SelectScratch& S, cudaStream_t st, const DedupSlot* table, uint64_t slots, Cand* out,
                       uint64_t cap) {
  if (S.stream != st) {
    S.release();
    S.stream = st;
  }
  auto* count = static_cast<unsigned long long*>(S.get(20, 8));
  SEL_CHECK(cudaMemsetAsync(count, 0, 8, st));
  const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>(blocks(slots, 256), 148u * 16u));
  if (slots) {
    k_compact_dedup<<<grid, 256, 0, st>>>(table, slots, out, cap, count);
    SEL_CHECK(cudaGetLastError());
  }
  unsigned long long n = 0;
  SEL_CHECK(cudaMemcpyAsync(&n, count, 8, cudaMemcpyDeviceToHost, st));
  SEL_CHECK(cudaStreamSynchronize(st));
  return n;
}

bool select_on_device(SelectScratch& S, cudaStream_t st, const RecordLayout& lay, const Cand* d_cands, uint64_t n64,
                      const std::vector<double>& levels, bool dedup, int64_t max_per_objective, uint64_t id_limit,
                      const Materializer& mat, SelectedSet& out) {
  out = SelectedSet{};
  if (S.stream != st) {  // buffers follow the stream they are used on
    S.release();
    S.stream = st;
  }
  if (n64 == 0 || levels.empty()) return true;
  if (n64 >= (1ull << 32)) return false;
  uint32_t lev_bits = 1;
  while ((1ull << lev_bits) < levels.size()) ++lev_bits;
  uint32_t id_bits = 1;
  while (id_bits < 64 && (id_limit >> id_bits) != 0) ++id_bits;
  if (id_bits + lev_bits > 63) return false;
  const uint32_t n = static_cast<uint32_t>(n64);
  const uint32_t nl = static_cast<uint32_t>(levels.size());
  std::vector<unsigned long long> keys_h(nl);
  for (uint32_t k = 0; k < nl; ++k) keys_h[k] = ord_bits(levels[k]);
  std::sort(keys_h.begin(), keys_h.end());
  auto* d_levels = static_cast<unsigned long long*>(S.get(18, size_t(nl) * 8));
  SEL_CHECK(cudaMemcpyAsync(d_levels, keys_h.data(), size_t(nl) * 8, cudaMemcpyHostToDevice, st));

  // 1. candidates at one of the levels
  auto* flag = static_cast<uint8_t*>(S.get(0, n));
  auto* iota = static_cast<uint32_t*>(S.get(1, size_t(n) * 4));
  auto* sel = static_cast<uint32_t*>(S.get(2, size_t(n) * 4));
  k_flag_levels<<<blocks(n, 256), 256, 0, st>>>(d_cands, n, d_levels, nl, flag, iota);
  SEL_CHECK(cudaGetLastError());
  const uint32_t m = select_flagged(S, st, iota, flag, sel, n);
  if (m == 0) return true;

  // 2. (level, id) order
  auto* key = static_cast<unsigned long long*>(S.get(3, size_t(m) * 8));
  auto* key_s = static_cast<unsigned long long*>(S.get(4, size_t(m) * 8));
  auto* pos = static_cast<uint32_t*>(S.get(5, size_t(m) * 4));
  auto* pos_s = static_cast<uint32_t*>(S.get(6, size_t(m) * 4));
  k_keys<<<blocks(m, 256), 256, 0, st>>>(d_cands, sel, m, d_levels, nl, id_bits, key, pos);
  SEL_CHECK(cudaGetLastError());
  sort_pairs(S, st, key, key_s, pos, pos_s, m, static_cast<int>(id_bits + lev_bits));

  // 3. systematic runs have no repeats: the per-objective cap applies before the records are rebuilt
  const uint32_t* order = nullptr;  // positions (in sorted order) of what is rebuilt
  uint32_t m1 = m;
  if (!dedup && max_per_objective >= 0) {
    auto* seq = static_cast<uint32_t*>(S.get(12, size_t(m) * 4));
    k_iota<<<blocks(m, 256), 256, 0, st>>>(m, seq);
    SEL_CHECK(cudaGetLastError());
    auto* fin = static_cast<uint32_t*>(S.get(14, size_t(m) * 4));
    m1 = cap_levels(S, st, seq, key_s, m, id_bits, nl, max_per_objective, fin);
    order = fin;
    if (m1 == 0) return true;
  }

  // 4. full records of the selected candidates, in (level, id) order
  auto* sc = static_cast<Cand*>(S.get(7, size_t(m1) * sizeof(Cand)));
  k_gather_cands<<<blocks(m1, 256), 256, 0, st>>>(d_cands, sel, pos_s, order, m1, sc);
  SEL_CHECK(cudaGetLastError());
  auto* recs = static_cast<uint8_t*>(S.get(19, size_t(m1) * lay.record_bytes));
  if (materialize(S, st, mat, sc, m1, recs) != 0)
    throw cuda_error("internal error: a rebuilt record's objective differs from the engine's");

  // 5. random mode: repeats, then the cap
  const uint32_t* fin_order = nullptr;
  uint32_t m2 = m1;
  if (dedup) {
    auto* hash = static_cast<unsigned long long*>(S.get(10, size_t(m1) * 8));
    auto* hs = key;   // the unsorted keys are no longer needed
    auto* q = pos;    // nor the unsorted positions
    auto* seq = static_cast<uint32_t*>(S.get(12, size_t(m1) * 4));
    k_hash<<<blocks(m1, 256), 256, 0, st>>>(recs, lay, m1, hash, seq);
    SEL_CHECK(cudaGetLastError());
    sort_pairs(S, st, hash, hs, seq, q, m1, 64);
    // records are in key_s order (no cap was applied before rebuilding): record p has key key_s[p]
    k_mark_repeats<<<blocks(m1, 256), 256, 0, st>>>(recs, lay, key_s, hs, q, m1, id_bits, flag);
    SEL_CHECK(cudaGetLastError());
    k_iota<<<blocks(m1, 256), 256, 0, st>>>(m1, seq);
    SEL_CHECK(cudaGetLastError());
    auto* kp = static_cast<uint32_t*>(S.get(15, size_t(m1) * 4));
    m2 = select_flagged(S, st, seq, flag, kp, m1);
    fin_order = kp;
    if (max_per_objective >= 0 && m2 > 0) {
      auto* fin = static_cast<uint32_t*>(S.get(14, size_t(m2) * 4));
      m2 = cap_levels(S, st, kp, key_s, m2, id_bits, nl, max_per_objective, fin);
      fin_order = fin;
    }
  }
  if (m2 == 0) return true;

  // 6. dense output arrays
  OutLayout o{};
  uint32_t sp_total = 0, sro_total = 0;
  for (uint32_t p = 0; p < lay.n_parts; ++p) {
    o.species_prefix[p] = sp_total;
    o.sro_prefix[p] = sro_total;
    sp_total += lay.n_sites[p];
    sro_total += lay.sro_bytes[p];
  }
  o.species_total = sp_total;
  o.sro_total = sro_total;
  const size_t b_obj = size_t(m2) * lay.tsz, b_sub = size_t(m2) * lay.n_parts * lay.tsz,
               b_sp = size_t(m2) * sp_total, b_sro = size_t(m2) * sro_total, b_id = size_t(m2) * 8;
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  auto* base = static_cast<uint8_t*>(S.get(3, al(b_obj) + al(b_sub) + al(b_sp) + al(b_sro) + al(b_id)));
  o.objective = base;
  o.sub_objective = o.objective + al(b_obj);
  o.species = o.sub_objective + al(b_sub);
  o.sro = o.species + al(b_sp);
  o.id = reinterpret_cast<unsigned long long*>(o.sro + al(b_sro));
  k_gather<<<blocks(uint64_t(m2) * 32, 256), 256, 0, st>>>(recs, lay, fin_order, m2, o);
  SEL_CHECK(cudaGetLastError());
  out.count = m2;
  out.objective.resize(b_obj);
  out.sub_objective.resize(b_sub);
  out.species.resize(b_sp);
  out.sro.resize(b_sro);
  out.id.resize(m2);
  copy_out(S, st, out.objective.data(), o.objective, b_obj);
  copy_out(S, st, out.sub_objective.data(), o.sub_objective, b_sub);
  copy_out(S, st, out.species.data(), o.species, b_sp);
  copy_out(S, st, out.sro.data(), o.sro, b_sro);
  copy_out(S, st, out.id.data(), o.id, b_id);
  SEL_CHECK(cudaStreamSynchronize(st));
  return true;
}

}  // namespace sqsg
