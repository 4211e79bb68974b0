// Device engine of the SQS optimisation: job/tile descriptors and the persistent tile kernel.
//
// One CTA of kBlock threads works on one tile at a time. A tile is a slice of one job's
// configuration space: in random mode kBlock independent shuffles per step, in systematic mode a
// contiguous interval of 1-based permutation ranks. Every thread owns one configuration at a time,
// stored as one byte per site in its own column of shared memory. Bond counting walks a per-shell,
// per-site grouped pair stream that every lane reads at the same address (a shared-memory
// broadcast), accumulates the species of the neighbours of site i in a packed register row, and adds
// the row to the lane's private histogram of ordered bond counts (s, species[i], species[j]) —
// exactly the counts of include/sqsgen/core/optimization.h:74-77. No global atomics in the loop.
#pragma once

#include <cstdint>
#include <cstring>

namespace sqsg {

// Order-preserving map of doubles onto unsigned 64-bit integers (for atomicMin).
__host__ __device__ __forceinline__ unsigned long long ord_bits(double x) {
#ifdef __CUDA_ARCH__
  unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
#else
  unsigned long long b;
  std::memcpy(&b, &x, 8);
#endif
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__host__ __device__ __forceinline__ double from_ord(unsigned long long u) {
  unsigned long long b = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
#ifdef __CUDA_ARCH__
  return __longlong_as_double(static_cast<long long>(b));
#else
  double x;
  std::memcpy(&x, &b, 8);
  return x;
#endif
}


// splitmix64 finalizer (Steele, Lea, Flood 2014): the per-id hash behind the order-independent level
// checksums.
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

constexpr int kBlock = 128;       // threads per CTA (each owns one configuration)
constexpr int kMinBlocks = 5;     // sqsg_engine_mask: CTAs per SM the register budget must allow (<= 102 registers)
constexpr int kK2MaxShells = 4;   // shells of the binary bit-mask path (per-shell counters in registers)
constexpr int kMinBlocksWide = 4; // sqsg_engine_wide (general path): 128 registers, no spills in the pair loop
constexpr int kMinBlocksLat = 2;   // sqsg_engine_lat (lattice path, up to 8 species): up to 255 registers
constexpr int kMinBlocksLat2 = 4;  // sqsg_engine_lat2 (lattice path, binary parts): up to 128 registers
constexpr int kMinBlocksLat5 = 3;  // sqsg_engine_lat5 (lattice path, up to 5 species): up to 168 registers
constexpr int kMinBlocksLatW = 2;  // sqsg_engine_latw (lattice path, 65-128 cells, up to 5 species)
constexpr int kMaxParts = 8;      // sublattices of a split-mode job
constexpr int kMaxWindows = 16;   // shuffle windows of an interact-mode job
constexpr int kMaxSpecies = 8;    // K per part handled by the packed-row counter
constexpr int kMaxGroup = 255;    // neighbours per (shell, site) group (8-bit row fields)
constexpr uint64_t kWaitNs = 2000000000ull;  // default bound of a staging wait (2 s of %globaltimer)
constexpr int kCtaLevelSlots = 64;       // per-CTA objective-level hash (shared memory)
constexpr int kLevelSlots = 4096;        // per-job objective-level hash (global memory)
constexpr int kMaxKeep = 1023;           // largest `keep` this build handles

// Counters of one job in device memory (unsigned long long each).
enum Counter : int {
  kCandidates = 0,  // candidate records appended (may exceed capacity: overflow)
  kThreshold = 1,   // ordered bits (double) of the search threshold, atomicMin
  kFinished = 2,    // configurations evaluated
  kError = 3,       // device error code (0 = none)
  kBest = 4,        // ordered bits (double) of the best objective seen, atomicMin
  kTilesDone = 5,   // tiles completed
  kLevelOverflow = 6,  // the job's level table ran out of slots
  kRecordsFull = 7,    // set once the candidate buffer is full (appends stop)
  kTilesLeft = 8,      // live queue: tiles of the job not yet finished
  kMismatch = 9,       // trace mode: lattice-path objectives that differ from the pair-stream path's
  kNumCounters = 16
};

enum DeviceError : unsigned long long { kErrNone = 0, kErrStageTimeout = 1, kErrBadJob = 2 };

// JobDesc::debug bits (set through sqsg_set_option, never by default).
enum DebugFlag : uint32_t {
  kDebugSkipStaging = 1u,  // expect the staged bytes but issue no copy: the staging wait runs out
};

// A candidate in the job's record buffer: the objective (as double: exact for float jobs too) and the
// configuration id. Configurations depend only on (job, id), so the full record (species, per-part
// objective, SRO) is rebuilt on the device for the selected candidates only (sqsg_materialize).
struct Cand {
  double objective;
  unsigned long long id;
};

// Distinct-configuration table of a random-mode re-run (JobDesc.dedup_slots > 0): open addressing on
// an exact configuration key (the multiset-permutation rank of the species, or the species bit mask
// of a binary bit-mask job), holding the smallest configuration id that produced the key and its
// objective. Empty slots have key == kDedupEmpty and id == ~0.
struct DedupSlot {
  unsigned long long key;
  unsigned long long id;
  double objective;
};
constexpr unsigned long long kDedupEmpty = ~0ull;
constexpr int kDedupProbes = 4096;
constexpr unsigned long long kDedupMaxSpace = 1ull << 40;  // rank arithmetic stays inside 64 bits

// One distinct objective value seen at or below the search threshold, with the number of
// evaluations that produced it and two order-independent 32-bit sums of hashes of their ids.
struct LevelSlot {
  unsigned long long key;    // ord_bits(objective as double); 0 = empty
  unsigned long long count;
  unsigned int sum_a, sum_b;
};

// One optimised structure: the whole cell in interact mode, one sublattice in split mode.
struct PartDesc {
  uint32_t n_sites, n_species, n_shells, n_windows;
  uint32_t hw;            // histogram words per (shell, species) row: ceil(K/2) 16-bit fields pairs
  uint32_t stream_words;  // words of the grouped pair stream
  uint32_t stream_narrow; // 1: 16-bit j offsets, two per word, one header word per group (N <= 512)
  uint32_t stream_global; // 1: the stream is read from the job blob (through L1), 0: staged in shared memory
  uint32_t blob_off;      // staged section: offset in the job blob (16-byte aligned)
  uint32_t static_bytes;  // staged section size (multiple of 16)
  uint32_t smem_off;      // part base in dynamic shared memory
  // offsets inside the staged section (identical in the blob and in shared memory)
  uint32_t cube_off;      // prefactors, pair weights, targets: 3 x S*K*K of T
  uint32_t win_off;       // 2 x n_windows u32 bounds [lo, hi), then n_windows u32 draw words (see shuffle_part)
  uint32_t stream_off;    // stream u32 words
  uint32_t species_off;   // N packed species codes (8 * species index)
  // shared-memory-only regions, relative to the part base
  uint32_t col_off;       // ceil(N/4) * kBlock words of species columns
  uint32_t hist_off;      // S*K*hw * kBlock words of histogram
  // candidate record layout
  uint32_t rec_species_off, rec_obj_off, rec_sro_off;
  // systematic mode: dense remap of the window values (core/shuffle.h:73-87)
  uint32_t unrank_k;
  uint32_t unrank_hist[kMaxSpecies];
  uint8_t unrank_rev[kMaxSpecies];
  // bond-trace layout
  uint32_t trace_species_off, trace_bonds_off;
  // binary fast path (K == 2, N <= 64): per (shell, site) neighbour masks, see run_tile_k2
  uint32_t k2_off;        // entries: uint4 {mask lo, mask hi, site | shell << 8, popcount}
  uint32_t k2_entries;
  uint32_t k2_shell_off;  // S x (pairs in shell, end of its entries, degree classes [begin, end),
                          //      degree sum of the largest class, 3 x 0)
  uint32_t k2_binom_off;  // blob offset (global, not staged) of C(m, j), m <= window, j <= ones
  uint32_t k2_nbp_off;    // neighbour masks by bit position: u32 [S][32] (N <= 32) or uint2 [S][64]
  uint32_t k2_zeros;      // 1: count over the zeros (species 0 is the minority), else over the ones
  // lattice path (a supercell whose pairs form whole translation classes, see run_tile_lat)
  uint32_t lat_km;        // 0: not on the lattice path; else the unrolled species count: K (K <= 5) or 8
  uint32_t lat_basis;     // unit-cell sites m
  uint32_t lat_cells;     // cells A*B*C (<= 128: one plane of lat_words words per unit-cell site and species)
  uint32_t lat_chunks;    // ceil(cells / 4)
  uint32_t lat_site_off;  // staged: u32 column offsets by (unit-cell site, cell), m x 4*chunks
  uint32_t lat_ent_off;   // staged: u32 classes  beta | beta2 << 4 | translation << 8, by shell
  uint32_t lat_shell_off; // staged: uint4 per shell (first class, first self-reverse class, end, pairs)
  uint32_t lat_tr_off;    // staged: LatTr per translation
  uint32_t lat_deg_off;   // staged: u32 shell-s neighbours of each unit-cell site, S x m
  uint32_t lat_planes_off;// shared-memory-only: per lane m x (K-1) one-hot planes of lat_words u64 (interleaved by lane)
  unsigned long long lat_full;     // the cells' bits (first word)
  unsigned long long lat_full_hi;  // cells 64..127 (two-word cell sets)
  // configuration keys of a deduplicating re-run: species counts of the part (all its sites), the
  // number of their distinct arrangements, and the product of the earlier parts' numbers
  uint32_t dd_counts[kMaxSpecies];
  unsigned long long dd_space;
  unsigned long long dd_stride;
  // reference-stream debug mode: random words one shuffle of the part draws (sum over windows of n_w - 1)
  uint32_t chain_draws;
  uint32_t ones;          // sites of species 1 (two-species parts: the binary path's minority count)
};

// A translation of the cell grid (bit c = x + A*(y + B*z)) by (dx, dy, dz), as rotations inside rows
// of A bits, blocks of A*B bits and the whole grid; a zero shift skips its stage. The masks have one
// 64-bit word per word of the job's cell sets (W = lat_words): the staged table holds LatTrW<W>.
template <int W> struct LatTrW {
  uint32_t sx, sxr, sy, syr, sz, szr, pad0, pad1;
  unsigned long long mxh[W], myh[W];  // cells whose source does not wrap in x, in y (the rest wrap)
};
using LatTr = LatTrW<2>;  // the host's working form (written out at the job's width)

struct JobDesc {
  uint32_t prec;          // 0 float, 1 double
  uint32_t mode;          // 0 random, 1 systematic
  uint32_t n_parts;
  uint32_t kw;            // 1: every part has K <= 4 (32-bit row), 2: K <= 8 (64-bit row)
  uint32_t k2;            // 0: general path; 1: binary bitmask path with N <= 32; 2: with N <= 64
  uint32_t keep;
  uint32_t record_bytes;  // bytes of a full (materialized) record; the engine itself writes Cand
  uint32_t smem_bytes;    // dynamic shared memory of the engine launch
  uint32_t smem_full;     // dynamic shared memory of the general layout (materialize, trace)
  uint32_t big_off;       // keep >= 32: per-warp best lists of big_len doubles at this offset
  uint32_t big_len;       // entries per warp list in shared memory (0: the list is one register per lane)
  uint32_t lat;           // 1: every part takes the lattice path
  uint32_t lat_kmax;      // lattice path: the largest unrolled species count (PartDesc.lat_km) of the parts
  uint32_t lat_words;     // lattice path: 64-bit words per cell set (1: up to 64 cells, 2: up to 128)
  uint32_t lat_pad2;
  uint32_t trace;         // 1: write every evaluated configuration to the trace buffers
  uint32_t trace_species_stride, trace_bonds_stride;
  uint64_t seed;
  uint64_t total;         // random: configurations; systematic: number of permutations
  const uint8_t* blob;
  uint8_t* records;
  uint64_t capacity;
  unsigned long long* counters;
  LevelSlot* levels;      // kLevelSlots
  uint8_t* trace_species;
  uint32_t* trace_bonds;
  void* trace_obj;
  uint64_t* trace_id;
  uint64_t trace_capacity;
  uint64_t trace_base;    // id of the first traced configuration
  uint64_t wait_ns;       // bound of the staging wait (%globaltimer nanoseconds)
  uint32_t debug;         // DebugFlag bits
  uint32_t reserved_dbg;
  DedupSlot* dedup;       // random-mode re-run: distinct-configuration table (null: candidates are appended)
  uint64_t dedup_mask;    // table slots - 1 (a power of two)
  // Reference-stream debug mode (random mode): configurations follow the reference's seeded
  // single-thread run, chained within the thread-pool blocks of [0, total) (see run_tile_chain).
  uint32_t chain;         // 1: this mode
  uint32_t chain_split;   // 1: split mode (shuffle, then evaluate); 0: interact (evaluate, then shuffle)
  uint64_t chain_blocks, chain_block, chain_rem;  // blocks, their base length, blocks one longer
  PartDesc parts[kMaxParts];
};

struct Tile {
  uint32_t job;         // index into the job table (a slot in live mode)
  uint32_t gen;         // live mode: generation of the job occupying the slot
  uint64_t start;       // random: index of the tile's first configuration; systematic: its 1-based rank
  uint64_t count;       // configurations in the tile (reference-stream mode: blocks, one per thread)
  uint64_t chain_configs;  // reference-stream mode: configurations of the tile's blocks (else unused)
};

// Queue control block of the persistent kernel, in device memory.
//  list mode (capacity == 0): tiles[0, n_tiles) are fixed; CTAs take them with atomicAdd on head.
//  live mode (capacity > 0): tiles is a ring the host appends to; the host's copy stream raises tail
//  after the tiles (and their jobs' descriptors) are in place, CTAs claim with atomicCAS on head and
//  leave after idle_limit empty polls (the host relaunches when new work arrives). With an owner
//  table, a CTA works only on an SM that the table gives to its ring and leaves (at start or
//  between tiles) once the SM belongs to another ring: the host partitions the SMs between rings
//  of different shared-memory sizes instead of letting their CTAs fragment every SM. alive[sm]
//  counts this ring's working CTAs per SM. A CTA that finds yield > 0 between tiles takes one
//  unit of it and leaves. launched - exited counts a ring's CTAs not yet gone.
struct QueueCtl {
  unsigned long long head;
  unsigned long long tail;
  unsigned int capacity;
  unsigned int idle_limit;
  unsigned int yield;
  unsigned int exited;
  unsigned int ring;
  unsigned int n_owner;                  // entries in owner[] (0: no owner table)
  const volatile unsigned char* owner;   // owner ring of each SM
  unsigned int* alive;                   // working CTAs of this ring per SM
  unsigned long long reserved;
};

}  // namespace sqsg
