// Host-side job preparation shared by every entry point (see prepare.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/sqsgen_b200.h"
#include "engine.cuh"

namespace sqsg {

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
// Byte offset of site x in a lane's species column (words of four sites interleaved across lanes).
inline uint32_t host_site_off(uint32_t x) { return (x >> 2) * (kBlock * 4) + (x & 3); }

struct PartMeta {
  uint32_t N, K, S;
};

struct PreparedJob {
  JobDesc desc{};               // device pointers filled at upload
  std::vector<uint8_t> blob;    // staged sections of all parts
  std::vector<PartMeta> parts;
  int prec = 1;
  bool systematic = false;
  uint64_t total = 0;           // configurations
  uint64_t keep = 1;
  int64_t max_rpo = -1;
  size_t record_bytes = 0;
  size_t tsz = 8;               // sizeof(T)
  uint32_t configs_per_thread = 1;
  uint64_t max_results = 0;     // caller's record capacity (0 = default)
  uint64_t range_first = 0, range_count = 0;  // share of the configuration space to evaluate
  // a re-run of an overflowed job: record capacity, starting threshold, passes already made
  uint64_t prepare_ns = 0;      // host time of prepare()
  uint64_t rerun_capacity = 0;
  double rerun_threshold = 0.0;
  int passes = 0;
};

// A job may have at most this many tiles (about 1.4e14 configurations at full-size tiles).
constexpr size_t kMaxJobTiles = 1u << 24;

// Validates the job and lays out its descriptor and blob (trace_capacity > 0: trace layout too).
PreparedJob prepare(const sqsg_job& job, uint64_t trace_capacity);
// Appends the job's tiles (guided sizes, at most max_per_thread configurations per thread).
void make_tiles(PreparedJob& pj, uint32_t job_index, std::vector<Tile>& tiles, uint64_t max_per_thread = 1u << 16);
// CTAs of the general-path kernel that fit on one SM of `device` with `dynamic_smem` bytes each.
int ctas_per_sm(int device, size_t dynamic_smem);

}  // namespace sqsg
