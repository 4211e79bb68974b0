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

// Launch choices of one job. Unset fields follow the fixed rules: the lattice path when the supercell
// hint holds, the pair stream staged in shared memory unless that costs a CTA per SM, as many CTAs per
// SM as fit, tiles of at most 65,536 configurations per thread. sqsg_autotune measures the choices
// for a job's bucket (job shape) and records the fastest; the shipped table holds measured entries.
struct Tuning {
  int path = -1;          // -1: rules; SQSG_PATH_GENERAL: the pair stream even when the lattice path applies
  int stage = -1;         // general path: -1 rules, 0 stream read through L1, 1 staged in shared memory
  uint32_t ctas = 0;      // CTAs per SM of a single-job launch (0: as many as fit)
  uint32_t tile_cap = 0;  // configurations per thread and tile, at most (0: 65,536)
};

// The bucket of a job's shape: precision, mode, parts, largest K and S, log2 of its sites and pairs,
// and whether it carries a supercell hint.
uint64_t bucket_key(const sqsg_job& job);
// The tuning for a bucket: measured in this process (sqsg_autotune), else the shipped table.
bool tuning_lookup(uint64_t key, Tuning& out);
void tuning_store(uint64_t key, const Tuning& t);

struct PartMeta {
  uint32_t N, K, S;
  uint32_t P;  // pairs
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
  Tuning tuning;                // launch choices (see Tuning)
  uint64_t rerun_capacity = 0;
  double rerun_threshold = 0.0;
  uint64_t rerun_slots = 0;     // > 0: the re-run collects distinct configurations in a table of this size
  int passes = 0;
  // random mode: configurations have exact keys (the parts' arrangement counts multiply to at most
  // kDedupMaxSpace = dedup_space), so a re-run may deduplicate on the device
  bool dedup_ok = false;
  uint64_t dedup_space = 0;
  // reference-stream debug mode (option "rapidrand", random jobs): the reference's thread-pool blocks
  // run as chains, one per thread (JobDesc.chain)
  bool chain = false;
};

// A job may have at most this many tiles (about 1.4e14 configurations at full-size tiles).
constexpr size_t kMaxJobTiles = 1u << 24;

// Validates the job and lays out its descriptor and blob (trace_capacity > 0: trace layout too).
// `tuning` (optional) overrides the table lookup for this job.
PreparedJob prepare(const sqsg_job& job, uint64_t trace_capacity, const Tuning* tuning = nullptr);
// Appends the job's tiles (guided sizes, at most max_per_thread configurations per thread).
void make_tiles(PreparedJob& pj, uint32_t job_index, std::vector<Tile>& tiles, uint64_t max_per_thread = 1u << 16);
// CTAs of the general-path kernel that fit on one SM of `device` with `dynamic_smem` bytes each.
int ctas_per_sm(int device, size_t dynamic_smem);

}  // namespace sqsg
