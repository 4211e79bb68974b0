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
  for (int k = 0; k < 16; ++k) {
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
    std::memcpy(static_cast<uint8_t*>(dst) + pend_off[k], S.bounce[k], pend_len[k]);
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

constexpr int kMaxLevels = 32;

struct Levels {
  unsigned long long key[kMaxLevels];  // ord_bits of the level values, ascending
  uint32_t n;
};

__device__ __forceinline__ double record_objective(const uint8_t* r, uint32_t tsz) {
  return tsz == 8 ? *reinterpret_cast<const double*>(r) : static_cast<double>(*reinterpret_cast<const float*>(r));
}

__device__ __forceinline__ int level_of(const Levels& L, unsigned long long key) {
  int lo = 0, hi = static_cast<int>(L.n) - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    if (L.key[mid] == key) return mid;
    if (L.key[mid] < key)
      lo = mid + 1;
    else
      hi = mid - 1;
  }
  return -1;
}

__global__ void k_flag_levels(const uint8_t* __restrict__ recs, uint32_t rb, uint32_t tsz, uint32_t n, Levels L,
                              uint8_t* __restrict__ flag, uint32_t* __restrict__ iota) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  flag[i] = level_of(L, ord_bits(record_objective(recs + static_cast<size_t>(i) * rb, tsz))) >= 0 ? 1 : 0;
  iota[i] = i;
}

__global__ void k_keys(const uint8_t* __restrict__ recs, RecordLayout lay, const uint32_t* __restrict__ sel,
                       uint32_t m, Levels L, uint32_t id_bits, bool with_hash, unsigned long long* __restrict__ key,
                       uint32_t* __restrict__ pos, unsigned long long* __restrict__ hash) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const uint8_t* r = recs + static_cast<size_t>(sel[j]) * lay.record_bytes;
  const int lev = level_of(L, ord_bits(record_objective(r, lay.tsz)));
  const unsigned long long id = *reinterpret_cast<const unsigned long long*>(r + 8);
  key[j] = (static_cast<unsigned long long>(lev) << id_bits) | id;
  pos[j] = j;
  if (with_hash) {
    unsigned long long h = 0xcbf29ce484222325ull;  // FNV-1a over the species bytes of all parts
    for (uint32_t p = 0; p < lay.n_parts; ++p)
      for (uint32_t x = 0; x < lay.n_sites[p]; ++x) h = (h ^ r[lay.species_off[p] + x]) * 0x100000001b3ull;
    hash[j] = h;
  }
}

__global__ void k_gather_hash(const unsigned long long* __restrict__ hash, const uint32_t* __restrict__ pos_s,
                              uint32_t m, unsigned long long* __restrict__ h2, uint32_t* __restrict__ iota) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  h2[p] = hash[pos_s[p]];
  iota[p] = p;
}

__device__ __forceinline__ bool same_species(const uint8_t* a, const uint8_t* b, const RecordLayout& lay) {
  for (uint32_t p = 0; p < lay.n_parts; ++p)
    for (uint32_t x = 0; x < lay.n_sites[p]; ++x)
      if (a[lay.species_off[p] + x] != b[lay.species_off[p] + x]) return false;
  return true;
}

// r runs over the (hash, level, id) order; q[r] is the (level, id) position. A record is a repeat
// when an earlier record of its hash run has the same level and the same species.
__global__ void k_mark_repeats(const uint8_t* __restrict__ recs, RecordLayout lay, const uint32_t* __restrict__ sel,
                               const uint32_t* __restrict__ pos_s, const unsigned long long* __restrict__ key_s,
                               const unsigned long long* __restrict__ h2s, const uint32_t* __restrict__ q, uint32_t m,
                               uint32_t id_bits, uint8_t* __restrict__ keep) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const uint32_t p = q[r];
  const unsigned long long lev = key_s[p] >> id_bits;
  const uint8_t* a = recs + static_cast<size_t>(sel[pos_s[p]]) * lay.record_bytes;
  bool repeat = false;
  for (uint32_t r2 = r; r2 > 0 && h2s[r2 - 1] == h2s[r]; --r2) {
    const uint32_t p2 = q[r2 - 1];
    if ((key_s[p2] >> id_bits) != lev) continue;
    if (same_species(recs + static_cast<size_t>(sel[pos_s[p2]]) * lay.record_bytes, a, lay)) {
      repeat = true;
      break;
    }
  }
  keep[p] = repeat ? 0 : 1;
}

__global__ void k_fill(uint8_t* __restrict__ v, uint32_t m, uint8_t value, uint32_t* __restrict__ iota) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  v[i] = value;
  iota[i] = i;
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

// One warp per selected record.
__global__ void k_gather(const uint8_t* __restrict__ recs, RecordLayout lay, const uint32_t* __restrict__ sel,
                         const uint32_t* __restrict__ pos_s, const uint32_t* __restrict__ order, uint32_t m,
                         OutLayout o) {
  const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (t >= m) return;
  const uint8_t* r = recs + static_cast<size_t>(sel[pos_s[order[t]]]) * lay.record_bytes;
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

}  // namespace

bool select_on_device(SelectScratch& S, cudaStream_t st, const RecordLayout& lay, const uint8_t* d_records,
                      uint64_t n64, const std::vector<double>& levels, bool dedup, int64_t max_per_objective,
                      uint64_t id_limit, SelectedSet& out) {
  out = SelectedSet{};
  if (S.stream != st) {  // buffers follow the stream they are used on
    S.release();
    S.stream = st;
  }
  if (n64 == 0 || levels.empty()) return true;
  if (levels.size() > static_cast<size_t>(kMaxLevels) || n64 >= (1ull << 32)) return false;
  uint32_t id_bits = 1;
  while (id_bits < 64 && (id_limit >> id_bits) != 0) ++id_bits;
  if (id_bits + 5 > 63) return false;
  const uint32_t n = static_cast<uint32_t>(n64);
  Levels L{};
  L.n = static_cast<uint32_t>(levels.size());
  for (size_t k = 0; k < levels.size(); ++k) L.key[k] = ord_bits(levels[k]);
  std::sort(L.key, L.key + L.n);

  // 1. records at one of the levels
  auto* flag = static_cast<uint8_t*>(S.get(0, n));
  auto* iota = static_cast<uint32_t*>(S.get(1, size_t(n) * 4));
  auto* sel = static_cast<uint32_t*>(S.get(2, size_t(n) * 4));
  k_flag_levels<<<blocks(n, 256), 256, 0, st>>>(d_records, lay.record_bytes, lay.tsz, n, L, flag, iota);
  SEL_CHECK(cudaGetLastError());
  const uint32_t m = select_flagged(S, st, iota, flag, sel, n);
  if (m == 0) return true;

  // 2. (level, id) order
  auto* key = static_cast<unsigned long long*>(S.get(3, size_t(m) * 8));
  auto* key_s = static_cast<unsigned long long*>(S.get(4, size_t(m) * 8));
  auto* pos = static_cast<uint32_t*>(S.get(5, size_t(m) * 4));
  auto* pos_s = static_cast<uint32_t*>(S.get(6, size_t(m) * 4));
  auto* hash = dedup ? static_cast<unsigned long long*>(S.get(7, size_t(m) * 8)) : nullptr;
  k_keys<<<blocks(m, 256), 256, 0, st>>>(d_records, lay, sel, m, L, id_bits, dedup, key, pos, hash);
  SEL_CHECK(cudaGetLastError());
  sort_pairs(S, st, key, key_s, pos, pos_s, m, static_cast<int>(id_bits + 5));

  // 3. repeats (random mode)
  auto* keep = flag;  // reused: one byte per (level, id) position
  uint32_t* iota2 = iota;
  if (dedup) {
    auto* h2 = static_cast<unsigned long long*>(S.get(10, size_t(m) * 8));
    auto* h2s = key;  // the unsorted keys are no longer needed
    auto* q = pos;    // nor the unsorted positions
    k_gather_hash<<<blocks(m, 256), 256, 0, st>>>(hash, pos_s, m, h2, iota2);
    SEL_CHECK(cudaGetLastError());
    sort_pairs(S, st, h2, h2s, iota2, q, m, 64);
    k_mark_repeats<<<blocks(m, 256), 256, 0, st>>>(d_records, lay, sel, pos_s, key_s, h2s, q, m, id_bits, keep);
    SEL_CHECK(cudaGetLastError());
  } else {
    k_fill<<<blocks(m, 256), 256, 0, st>>>(keep, m, 1, iota2);
    SEL_CHECK(cudaGetLastError());
  }
  auto* kp = static_cast<uint32_t*>(S.get(12, size_t(m) * 4));
  uint32_t m2 = select_flagged(S, st, iota2, keep, kp, m);

  // 4. per-objective cap
  const uint32_t* order = kp;
  if (max_per_objective >= 0 && m2 > 0) {
    auto* start = static_cast<uint32_t*>(S.get(13, kMaxLevels * 4));
    auto* cflag = static_cast<uint8_t*>(S.get(11, m2));
    auto* fin = static_cast<uint32_t*>(S.get(14, size_t(m2) * 4));
    SEL_CHECK(cudaMemsetAsync(start, 0, kMaxLevels * 4, st));
    k_level_starts<<<blocks(m2, 256), 256, 0, st>>>(kp, key_s, m2, id_bits, start);
    SEL_CHECK(cudaGetLastError());
    k_cap<<<blocks(m2, 256), 256, 0, st>>>(kp, key_s, m2, id_bits, start,
                                           static_cast<unsigned long long>(max_per_objective), cflag);
    SEL_CHECK(cudaGetLastError());
    m2 = select_flagged(S, st, kp, cflag, fin, m2);
    order = fin;
  }
  if (m2 == 0) return true;

  // 5. dense output arrays
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
  auto* base = static_cast<uint8_t*>(S.get(15, al(b_obj) + al(b_sub) + al(b_sp) + al(b_sro) + al(b_id)));
  o.objective = base;
  o.sub_objective = o.objective + al(b_obj);
  o.species = o.sub_objective + al(b_sub);
  o.sro = o.species + al(b_sp);
  o.id = reinterpret_cast<unsigned long long*>(o.sro + al(b_sro));
  k_gather<<<blocks(uint64_t(m2) * 32, 256), 256, 0, st>>>(d_records, lay, sel, pos_s, order, m2, o);
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
