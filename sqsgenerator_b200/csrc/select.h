// Result-set selection on the device: from a job's candidate records to the reference's result
// set (every distinct configuration whose objective is one of the keep+1 best distinct objectives,
// ordered by objective then id, at most max_results_per_objective+1 per objective).
#pragma once

#include <cuda_runtime.h>

#include <sys/mman.h>

#include <cstdint>
#include <cstdlib>
#include <memory>
#include <new>
#include <utility>
#include <vector>

#include "engine.cuh"

namespace sqsg {

// Where the fields of one candidate record live (offsets in bytes inside a record).
struct RecordLayout {
  uint32_t record_bytes = 0;
  uint32_t tsz = 8;  // sizeof(T)
  uint32_t n_parts = 1;
  uint32_t obj_off[kMaxParts] = {};
  uint32_t species_off[kMaxParts] = {};
  uint32_t n_sites[kMaxParts] = {};
  uint32_t sro_off[kMaxParts] = {};
  uint32_t sro_bytes[kMaxParts] = {};
};

// Allocator for result arrays of up to millions of configurations: resize() leaves new elements
// uninitialised (they are overwritten right away; zero-filling first doubled the cost), and blocks
// of 64 MiB and more are 2 MiB-aligned and advised for transparent huge pages, so that filling
// them takes a few thousand page faults instead of a million.
template <class T> struct NoInitAlloc : std::allocator<T> {
  static constexpr size_t kHuge = 2u << 20, kLarge = 64u << 20;
  template <class U> struct rebind { using other = NoInitAlloc<U>; };
  NoInitAlloc() = default;
  template <class U> NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
  T* allocate(size_t n) {
    const size_t bytes = n * sizeof(T);
    if (bytes < kLarge) return std::allocator<T>::allocate(n);
    const size_t rounded = (bytes + kHuge - 1) / kHuge * kHuge;
    void* p = std::aligned_alloc(kHuge, rounded);
    if (!p) throw std::bad_alloc();
    madvise(p, rounded, MADV_HUGEPAGE);
    return static_cast<T*>(p);
  }
  void deallocate(T* p, size_t n) noexcept {
    if (n * sizeof(T) < kLarge)
      std::allocator<T>::deallocate(p, n);
    else
      std::free(p);
  }
  template <class U> void construct(U* p) noexcept { ::new (static_cast<void*>(p)) U; }
  template <class U, class... A> void construct(U* p, A&&... a) { ::new (static_cast<void*>(p)) U(std::forward<A>(a)...); }
};
using ByteVec = std::vector<uint8_t, NoInitAlloc<uint8_t>>;
using IdVec = std::vector<uint64_t, NoInitAlloc<uint64_t>>;

struct SelectedSet {
  uint64_t count = 0;
  ByteVec objective, sub_objective, species, sro;  // raw T bytes / species bytes
  IdVec id;
};

// Grow-only device scratch for select_on_device, bound to the stream it was last used on.
struct SelectScratch {
  static constexpr int kSlots = 21;
  void* buf[kSlots] = {};
  size_t size[kSlots] = {};
  cudaStream_t stream = nullptr;
  uint8_t* bounce[2] = {};        // pinned host buffers for large device-to-host copies
  cudaEvent_t bounce_done[2] = {};
  ~SelectScratch() { release(); }
  void* get(int slot, size_t bytes);
  // Frees every buffer on its stream and waits for it; call before that stream is destroyed.
  void release();
};

// Rebuilds full records of selected candidates on the device (sqsg_materialize) for one job.
struct Materializer {
  JobDesc job;        // the job's descriptor with device pointers (uploaded by materialize)
  size_t smem = 0;    // dynamic shared memory of the launch (the job's general layout)
};

// Launches sqsg_materialize for m candidates (device array, in selection order) into m full records
// at d_out, on `stream`; returns the number of objective mismatches (0 unless the engine is wrong),
// after waiting for the stream. Scratch slots 16 and 17 of S hold the descriptor and the counter.
uint64_t materialize(SelectScratch& S, cudaStream_t stream, const Materializer& mat, const Cand* d_cands, uint32_t m,
                     uint8_t* d_out);

// Gathers the occupied slots of a distinct-configuration table (a deduplicating re-run) into
// candidates at `out` (at most cap, in no particular order) and returns how many slots were occupied,
// after waiting for the stream. Scratch slot 20 of S holds the counter.
uint64_t compact_dedup(SelectScratch& S, cudaStream_t stream, const DedupSlot* table, uint64_t slots, Cand* out,
                       uint64_t cap);

// Selects, from n device-resident candidates, those whose objective equals one of `levels` (the
// keep+1 smallest distinct objectives, exact), orders them by (objective, id), rebuilds their full
// records, and (random runs, dedup) keeps among equal species the record with the smallest id, then at
// most max_per_objective+1 per objective. Returns false without doing anything when the ids do not
// leave room for the level index in a 64-bit sort key; the caller then selects on the host.
bool select_on_device(SelectScratch& scratch, cudaStream_t stream, const RecordLayout& layout, const Cand* d_cands,
                      uint64_t n, const std::vector<double>& levels, bool dedup, int64_t max_per_objective,
                      uint64_t id_limit, const Materializer& mat, SelectedSet& out);

}  // namespace sqsg
