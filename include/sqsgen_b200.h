/*
 * sqsgen_b200 — C ABI of the B200-native SQS optimisation hot path.
 *
 * The library replaces the optimisation loop of dgehringer/sqsgenerator 0.5.6 (a header-only C++
 * library with no C ABI of its own). Each entry point below names the reference interface it
 * replaces (paths relative to the reference repository root).
 *
 * Conventions
 *  - Plain C types, caller-owned buffers, no exceptions across the ABI: every call returns an
 *    sqsg_status; sqsg_last_error() gives the message of the calling thread's last failure.
 *  - prec selects the floating type of every `void*` array: 0 = float (single), 1 = double.
 *  - Cubes (prefactors, pair weights, targets, SRO) are row-major [shell][a][b] over dense species
 *    indices (sorted atomic numbers), shells packed by ascending shell index.
 *  - Species arrays passed to the optimiser are "packed": values 0..K-1 in the sorted site order
 *    produced by the host precompute (sqsg_sort_by_sublattice).
 *  - The optimiser runs on one CUDA device per call; calls on different host threads with different
 *    jobs may run concurrently. There is no CPU fallback: without a usable CUDA device the
 *    optimiser returns SQSG_ERR_CUDA.
 */
#ifndef SQSGEN_B200_H
#define SQSGEN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SQSG_ABI_VERSION 2

typedef enum {
  SQSG_OK = 0,
  SQSG_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
  SQSG_ERR_OUT_OF_RANGE = 2,     /* std::out_of_range in the reference */
  SQSG_ERR_CAPACITY = 3,         /* caller buffer too small; the needed size is reported */
  SQSG_ERR_CUDA = 4,             /* CUDA runtime failure or no device */
  SQSG_ERR_UNSUPPORTED = 5,      /* a size this build does not handle (message says which) */
  SQSG_ERR_TIMEOUT = 6,          /* a bounded device wait ran out */
  SQSG_ERR_BUSY = 7              /* server queue full / admission refused */
} sqsg_status;

enum { SQSG_PREC_SINGLE = 0, SQSG_PREC_DOUBLE = 1 };
enum { SQSG_ITERATION_RANDOM = 0, SQSG_ITERATION_SYSTEMATIC = 1 };
enum { SQSG_SUBLATTICE_INTERACT = 0, SQSG_SUBLATTICE_SPLIT = 1 };
enum { SQSG_TIMING_TOTAL = 0, SQSG_TIMING_CHUNK_SETUP = 1, SQSG_TIMING_LOOP = 2, SQSG_TIMING_COMM = 3 };

/* ------------------------------------------------------------------------------------------------
 * Library information
 */
const char* sqsg_version(void);
/* Copies the calling thread's last error message (NUL-terminated, truncated to len). */
size_t sqsg_last_error(char* buf, size_t len);
/* Number of CUDA devices visible to the library (0 when none). */
int sqsg_device_count(void);

/* ------------------------------------------------------------------------------------------------
 * Host precompute: geometry, shells, prefactors, pair list (run once per job, on the CPU).
 */

/* core::structure::supercell — include/sqsgen/core/structure.h:335-366.
 * lattice: 3x3 row-major (rows are lattice vectors); frac: n x 3. Outputs hold a*b*c*n sites. */
sqsg_status sqsg_supercell(int prec, const void* lattice, const void* frac, const uint8_t* species,
                           uint32_t n, uint32_t a, uint32_t b, uint32_t c, void* lattice_out,
                           void* frac_out, uint8_t* species_out);

/* core::detail::distance_matrix — include/sqsgen/core/structure.h:35-69 (minimum over the 27
 * images (-1,0,1)^3). out: n x n row-major. */
sqsg_status sqsg_distance_matrix(int prec, const void* lattice, const void* frac, uint32_t n, void* out);

/* core::detail::shell_matrix — include/sqsgen/core/structure.h:71-100. radii[0] must be 0. */
sqsg_status sqsg_shell_matrix(int prec, const void* distances, uint32_t n, const void* radii,
                              uint32_t n_radii, double atol, double rtol, uint32_t* out);

/* core::distances_naive — include/sqsgen/core/structure.h:195-207.
 * *n_out: in = capacity of out, out = number of radii (SQSG_ERR_CAPACITY if it did not fit). */
sqsg_status sqsg_distances_naive(int prec, const void* distances, uint32_t n, double atol, double rtol,
                                 void* out, uint32_t* n_out);

/* core::distances_histogram — include/sqsgen/core/structure.h:209-258 (peak detection). */
sqsg_status sqsg_distances_histogram(int prec, const void* distances, uint32_t n, double bin_width,
                                     double peak_isolation, void* out, uint32_t* n_out);

/* core::detail::compute_prefactors — include/sqsgen/core/structure.h:136-192.
 * shells: n x n shell matrix; shell_ids: the weighted shells (ascending); species: atomic numbers.
 * out: S x K x K row-major, K = distinct species. */
sqsg_status sqsg_prefactors(int prec, const uint32_t* shells, uint32_t n, const uint32_t* shell_ids,
                            uint32_t n_shells, const uint8_t* species, void* out);

/* core::structure::pairs — include/sqsgen/core/structure.h:434-451 (i < j, packed shell index).
 * *n_pairs: in = capacity (in pairs), out = count. pairs_out: 3 x count (i, j, shell). */
sqsg_status sqsg_pairs(const uint32_t* shells, uint32_t n, const uint32_t* shell_ids, uint32_t n_shells,
                       uint32_t* pairs_out, uint32_t* n_pairs);

/* optimization::compute_shuffling_bounds — include/sqsgen/core/optimization.h:35-72.
 * sublattice_of_site[i] = index of the sublattice containing site i, or n_sublattices when none.
 * Writes sort_order (n; sorted position -> original site) and windows (2 x *n_windows). */
sqsg_status sqsg_sort_by_sublattice(const uint32_t* sublattice_of_site, uint32_t n, uint32_t n_sublattices,
                                    uint32_t* sort_order, uint32_t* windows, uint32_t* n_windows);

/* ------------------------------------------------------------------------------------------------
 * Multiset permutations (u64 ranks; the reference parser rejects counts above u64,
 * include/sqsgen/io/config/combined.h:88-95).
 */
/* core::num_permutations — include/sqsgen/core/permutation.h:17-32. SQSG_ERR_OUT_OF_RANGE on overflow. */
sqsg_status sqsg_num_permutations(const uint8_t* conf, uint32_t n, uint64_t* out);
/* core::rank_permutation — include/sqsgen/core/permutation.h:34-50 (1-based, dense values). */
sqsg_status sqsg_rank_permutation(const uint8_t* conf, uint32_t n, uint64_t* rank);
/* core::unrank_permutation — include/sqsgen/core/permutation.h:52-78 (writes dense values). */
sqsg_status sqsg_unrank_permutation(uint8_t* conf, uint32_t n, uint64_t rank);

/* ------------------------------------------------------------------------------------------------
 * The optimiser — replaces sqsgen::run_optimization (include/sqsgen/sqs.h:625-634) and its worker
 * loop optimizer<T,IterationMode,SublatticeMode>::run (include/sqsgen/sqs.h:299-580).
 */
typedef struct {
  uint32_t n_sites;           /* N: sites of this optimised structure, sorted order */
  uint32_t n_species;         /* K */
  uint32_t n_shells;          /* S */
  uint32_t n_pairs;           /* P */
  uint32_t n_windows;         /* shuffle windows (interact: one per sublattice) */
  uint32_t reserved;
  const uint32_t* pairs;      /* 3 x P: (i, j, shell), i < j */
  const uint8_t* species;     /* N packed species (0..K-1) */
  const uint32_t* windows;    /* 2 x n_windows: [lo, hi) */
  const void* prefactors;     /* S x K x K */
  const void* pair_weights;   /* S x K x K, already multiplied by the shell weights */
  const void* target;         /* S x K x K */
  /* Optional supercell hint (NULL: none). When the structure is a supercell of cells[0] x cells[1] x
   * cells[2] copies of a unit cell, lattice holds per site (sorted order) 4 values: the index of its
   * unit-cell site among this structure's unit-cell sites (0..n_basis-1) and its cell indices along
   * the three lattice vectors. The library checks the hint against the pair list: when every shell's
   * pairs are whole translation classes it counts bonds with translated bit planes (SQSG_PATH_LATTICE,
   * up to 64 cells, or up to 128 cells with at most five species); otherwise the hint is ignored.
   * Results do not depend on it. */
  const uint32_t* lattice;
  uint32_t cells[3];
  uint32_t n_basis;
} sqsg_sublattice;

typedef struct {
  uint64_t finished;          /* configurations evaluated */
  uint64_t working;           /* configurations in flight */
  uint64_t best_rank;         /* systematic: rank of the best; random: its configuration index */
  double best_objective;
  uint64_t timings_ns[4];     /* SQSG_TIMING_* */
} sqsg_statistics;

/* Progress callback, invoked from the calling host thread (never from device code) while the
 * device works. Return non-zero to stop early (like sqs_callback_context::stop, types.h:222-232);
 * results found so far are kept. */
typedef int (*sqsg_callback)(const sqsg_statistics* stats, void* user);

typedef struct {
  int32_t prec;
  int32_t iteration_mode;
  int32_t sublattice_mode;
  uint32_t n_sublattices;     /* interact: 1 (windows carry the sublattices); split: one per sublattice */
  const sqsg_sublattice* sublattices;
  uint64_t iterations;        /* random: configurations to evaluate; systematic: 0 = all permutations */
  uint64_t chunk_size;        /* progress-callback granularity in configurations (0: default); the
                                 reference's block size in the "rapidrand" debug mode */
  uint64_t keep;              /* the reference's `keep` (1..1023 in this build) */
  int64_t max_results_per_objective; /* < 0: unset */
  uint64_t seed;              /* random mode: key of the Philox4x32-10 blocks that seed each configuration's
                                 shuffle words (rapidrand seed in the "rapidrand" debug mode) */
  int32_t has_seed;           /* 0: a random seed is drawn */
  int32_t device;             /* CUDA device ordinal */
  const volatile int32_t* cancel; /* optional: set non-zero from any thread to stop early */
  sqsg_callback callback;     /* optional */
  void* user;
  uint64_t max_results;       /* record capacity of the result set (0: library default, grown on demand
                                 within a 4 GiB device budget) */
  uint64_t range_first;       /* evaluate only configurations [range_first, range_first + range_count) of the */
  uint64_t range_count;       /* job (0 = to the end): one GPU's share, like optimizer_base::iteration_range
                                 (include/sqsgen/sqs.h:226-238). Systematic: rank range_first+1 onwards. */
} sqsg_job;

typedef struct sqsg_run sqsg_run;

/* Runs one job to completion on job->device and returns its result set in *run (free with
 * sqsg_run_free). The result set is every distinct configuration whose objective is within the
 * keep+1 best distinct objectives seen — the configurations the reference's result collection
 * (include/sqsgen/core/results.h:42-99, sqs.h:421-438) always returns — capped at
 * max_results_per_objective+1 per objective when that is set. */
sqsg_status sqsg_optimize(const sqsg_job* job, sqsg_run** run);

/* Result access. Records are sorted by total objective, then by id. */
uint64_t sqsg_run_count(const sqsg_run* run);
/* Copies records [first, first+n). Any output pointer may be NULL. Per record: objective (prec),
 * sub_objectives (n_sublattices, prec), species (sum of N, packed, sorted order), sro
 * (sum of S*K*K, prec, row-major), id (systematic: 1-based rank; random: 0-based configuration index;
 * configuration i is the (i - c)-th shuffle of the chain that starts at index c). */
sqsg_status sqsg_run_copy(const sqsg_run* run, uint64_t first, uint64_t n, void* objective,
                          void* sub_objectives, uint8_t* species, void* sro, uint64_t* id);
sqsg_status sqsg_run_statistics(const sqsg_run* run, sqsg_statistics* stats);
void sqsg_run_free(sqsg_run* run);

/* The keep+1 best distinct objectives seen (ascending), each with the number of evaluations that
 * produced it and an order-independent checksum of their ids (two 32-bit sums of splitmix64(id),
 * low and high halves). These are exact even when the record set was cut at its capacity.
 * *n: in = capacity, out = number of levels. No reference counterpart (the reference keeps every
 * record); they make results of any size comparable. */
sqsg_status sqsg_run_levels(const sqsg_run* run, uint32_t* n, double* values, uint64_t* counts,
                            uint64_t* checksums);
/* candidates: records the device appended; truncated: 1 when the record set hit its capacity;
 * levels_exact: 0 when the level table overflowed (then only the records define the result). */
sqsg_status sqsg_run_info(const sqsg_run* run, uint64_t* candidates, int32_t* truncated, int32_t* levels_exact);
/* Host-side time of the stages of the call that produced the run, in nanoseconds (*n: in =
 * capacity, out = SQSG_STAGE_COUNT): job preparation and tiling; uploads; the engine kernel (CUDA
 * events); the host's wait for it (kernel time plus launch and queueing); counters and objective
 * levels downloaded and assessed; result-set selection (device selection, record rebuilding and the
 * copy into host memory); and the whole call. Stages of the served form are not recorded (zeros).
 * No reference counterpart. */
enum {
  SQSG_STAGE_PREPARE = 0, SQSG_STAGE_UPLOAD = 1, SQSG_STAGE_KERNEL = 2, SQSG_STAGE_WAIT = 3,
  SQSG_STAGE_LEVELS = 4, SQSG_STAGE_SELECT = 5, SQSG_STAGE_TOTAL = 6, SQSG_STAGE_COUNT = 7
};
sqsg_status sqsg_run_stages(const sqsg_run* run, uint64_t* ns, uint32_t* n);
/* Bytes the call copied host->device (job blob, tiles, descriptors) and device->host (records,
 * level table, counters). */
sqsg_status sqsg_run_transfer(const sqsg_run* run, uint64_t* h2d_bytes, uint64_t* d2h_bytes);

/* Debug/parity trace: like sqsg_optimize, but additionally records every evaluated configuration
 * (at most `capacity`; SQSG_ERR_CAPACITY otherwise) with its packed species, ordered bond counts
 * (S x K x K u32 per sublattice, like core/optimization.h:74-77) and objective. Sizes: species
 * capacity x sum N; bonds capacity x sum S*K*K; objective capacity (prec); id capacity. */
sqsg_status sqsg_optimize_trace(const sqsg_job* job, sqsg_run** run, uint64_t capacity, uint64_t* count,
                                uint8_t* species, uint32_t* bonds, void* objective, uint64_t* id);

/* ------------------------------------------------------------------------------------------------
 * Options and launch plans (no reference counterpart: the reference's only knobs are the thread
 * count and chunk size, include/sqsgen/io/config/combined.h:122-136).
 *
 * Process-wide options, read when a job is prepared:
 *   "force_general"      0/1   1: every job takes the general pair-stream path (the bit-mask path is
 *                              skipped); results are identical, only the speed differs.
 *   "stage_wait_ns"      > 0   bound of the device's wait for a job's staged data (default 2e9).
 *   "debug_skip_staging" 0/1   debug: the device expects the staged data but no copy is issued, so
 *                              that the bounded wait runs out and the call returns SQSG_ERR_TIMEOUT.
 *   "use_tuning"         0/1   1 (default): jobs take the measured launch choices of their bucket
 *                              (sqsg_autotune, shipped table); 0: the fixed rules.
 *   "default_candidates" > 0   candidate capacity (16-byte entries) of a job that leaves max_results
 *                              at 0 (default 2^20); a job that overflows it runs again (below).
 *   "rerun_record_bytes" > 0   bytes of full records that the re-run of an overflowed job may produce
 *                              (default 4 GiB). The re-run stores every evaluation at or below the
 *                              final (keep+1)-th best objective T*; when those are too many, a random
 *                              job whose configurations have exact keys (the arrangements of its
 *                              species multisets number at most 2^40) stores each distinct
 *                              configuration once, with its smallest id. Otherwise the result set is
 *                              truncated (sqsg_run_info) and the objective levels stay exact.
 *   "rapidrand"          0/1   debug (default 0): random jobs follow the reference's seeded
 *                              single-thread run (core/shuffle.h:23-50 with rapidhash's rapidrand,
 *                              blocks of chunk_size, sqs.h:348-466) instead of this library's stream; each
 *                              block runs as one chain on one GPU thread, so a job has only
 *                              iterations / chunk_size-way parallelism. Configuration ids are the
 *                              reference's iteration indices. Pair-stream path only; sqsg_optimize,
 *                              sqsg_optimize_batch and traces only (not the server, not ranges).
 *   "server_finalizers"  > 0   result-selection threads of servers created afterwards (default 4).
 *   "binary_floyd"       0/1   1 (default): in random mode a shuffle window that holds exactly two
 *                              species draws the sites of its rarer species (Floyd's sampling: m
 *                              draws for m such sites) instead of n - 1 Fisher-Yates swaps; both give
 *                              every arrangement of the window the same probability. 0: Fisher-Yates
 *                              on every window. Read when a job is prepared; it selects the stream,
 *                              so results of one seed differ between the two settings.
 * Unknown names give SQSG_ERR_INVALID_ARGUMENT. */
sqsg_status sqsg_set_option(const char* name, int64_t value);
sqsg_status sqsg_get_option(const char* name, int64_t* value);

enum { SQSG_PATH_GENERAL = 0, SQSG_PATH_BITMASK = 1, SQSG_PATH_LATTICE = 2 };

typedef struct {
  int32_t path;           /* SQSG_PATH_* */
  int32_t stream_narrow;  /* general path: 16-bit neighbour offsets (sites <= 512) */
  int32_t stream_staged;  /* general path: pair stream staged in shared memory (0: read through L1) */
  uint32_t lattice_units; /* lattice path: 64-bit AND-popcount units per configuration (translation
                             classes x species pairs a <= b < K-1); 0 on the other paths */
} sqsg_part_plan;

typedef struct {
  uint32_t n_parts;
  uint32_t smem_bytes;    /* dynamic shared memory per CTA */
  uint32_t ctas_per_sm;   /* resident CTAs per SM (0 when no device is visible) */
  uint32_t record_bytes;  /* bytes per candidate record in device memory */
  char kernel[32];        /* the engine kernel a sqsg_optimize call launches */
  sqsg_part_plan parts[8];
  uint64_t bucket;        /* the job's bucket in the tuning table (see sqsg_autotune) */
  int32_t tuned;          /* 1 when the launch follows a measured tuning entry */
  uint32_t shuffle_draws; /* random mode: bounded draws per configuration over all parts (a window of
                             two species draws its rarer species' sites, option "binary_floyd";
                             another window n - 1); 0 in systematic mode */
} sqsg_plan;

/* How sqsg_optimize would run the job: per optimised structure the evaluation path, and the launch
 * shape. Validates the job like sqsg_optimize; needs no device (ctas_per_sm is then 0). */
sqsg_status sqsg_plan_job(const sqsg_job* job, sqsg_plan* plan);

/* Launch choices of one job bucket (sqsg_autotune). */
typedef struct {
  int32_t path;           /* SQSG_PATH_* */
  int32_t stream_staged;  /* general path: 1 pair stream staged in shared memory, 0 read through L1 */
  uint32_t ctas_per_sm;   /* CTAs per SM of the launch (0: as many as fit) */
  uint32_t tile_cap;      /* configurations per thread and tile, at most */
  double configs_per_s;   /* measured engine rate (kernel time) */
} sqsg_tuning;

/* Autotuner (no reference counterpart; the reference's only scheduling knob is the chunk size,
 * include/sqsgen/io/config/combined.h:122-136). Times short prefixes of the job on its device for each
 * launch choice that applies to it — evaluation path (lattice or pair stream), pair-stream staging,
 * CTAs per SM, tile size — within about `seconds`, and records the fastest for the job's bucket (its
 * precision, mode, parts, species, shells, and the powers of two of its sites and pairs). Later jobs of
 * the same bucket in this process take the recorded choices (option "use_tuning", default 1); the
 * library also ships a table measured on a B200. Results never depend on the choices. *best: the
 * chosen; tried (optional, capacity *n_tried, out = count): every choice measured. */
sqsg_status sqsg_autotune(const sqsg_job* job, double seconds, sqsg_tuning* best, sqsg_tuning* tried,
                          uint32_t* n_tried);

/* Peak-rate microbenchmarks used as roofline denominators (no reference counterpart).
 * kind 0: shared-memory load bandwidth (bytes/s); kind 1: 32-bit integer lane operations per second;
 * kind 2: 32-bit population counts per second, each with the logic op and the add that the lattice
 * path pairs with it. */
sqsg_status sqsg_microbench(int kind, int device, double* rate, double* seconds);

/* Allocation-free variant of sqsg_optimize, for callers that cannot allocate device memory (a host
 * framework that owns the whole device budget through its own pool, a process whose memory is capped
 * once work starts). No counterpart in the reference. It runs the same engine kernel, but all of its
 * device scratch lives in one static __device__ array of about 3.6 MiB that every GPU loading this
 * library holds until exit, and it calls no cudaMalloc/cudaFree or other allocating routine.
 * Outputs: the keep+1 best objectives with exact counts and id checksums (*n_levels: in = capacity,
 * out = count) — the values sqsg_run_levels gives for the same job — and, of the statistics, finished,
 * best_objective and the total/loop timings; best_rank is set to UINT64_MAX (not reported: no
 * configuration records are kept). A job with more distinct objectives than the 4096-slot level table
 * takes before the search threshold settles runs again from a tighter threshold (at most 8 passes;
 * SQSG_ERR_CAPACITY if the table still overflows); the timings cover every pass.
 * Limits: staged job data <= 3 MiB, <= 16448 tiles; no callback or
 * cancellation; `stream` may be NULL (legacy default stream). The first call on a device looks up the
 * array's device address, so make it before any stream capture. Calls share the array: each call
 * resets what must start at zero, calls from one process are serialised by a lock, and a call returns
 * only after its kernel has finished, also on error paths. Separate processes each have their own copy
 * of the array. Work of this process that still uses the array on the GPU when another call starts
 * (which the lock and the wait above rule out for this entry point's own calls) would race with it.
 * Messages go to err. */
sqsg_status sqsg_optimize_levels_noalloc(const sqsg_job* job, void* stream, uint32_t* n_levels, double* values,
                                         uint64_t* counts, uint64_t* checksums, sqsg_statistics* stats, char* err,
                                         size_t err_len);

/* ------------------------------------------------------------------------------------------------
 * Batched form: many independent jobs in one persistent launch fed by a device tile queue
 * (no reference counterpart; the reference runs one configuration per call).
 */
sqsg_status sqsg_optimize_batch(const sqsg_job* jobs, uint32_t n_jobs, sqsg_run** runs);

/* ------------------------------------------------------------------------------------------------
 * Served form: continuous batching (no reference counterpart). Jobs submitted while others run are
 * admitted as job slots, ring space and device memory (data + records: the job's footprint) free up;
 * their tiles join a persistent kernel that is already running. A job's result is the same as from
 * sqsg_optimize: it depends only on the job.
 */
typedef struct sqsg_server sqsg_server;

typedef struct {
  int32_t device;
  uint32_t max_jobs;              /* jobs admitted at once (0: 256) */
  uint64_t arena_bytes;           /* device memory for admitted jobs' data and records (0: 16 GiB, at most 1/4 of free memory) */
  uint64_t default_max_results;   /* record capacity of a job that leaves max_results at 0 (0: 65536) */
} sqsg_server_options;

typedef struct {
  uint64_t submitted, admitted, completed, pending, active;
  uint64_t configurations;        /* evaluated by completed jobs */
  uint64_t launches;              /* persistent-kernel launches so far */
  uint64_t arena_free_bytes;
} sqsg_server_counters;

sqsg_status sqsg_server_create(const sqsg_server_options* options, sqsg_server** server);
/* Validates and prepares the job on the calling thread and queues it; returns at once with a ticket.
 * Jobs with a callback or cancel flag are rejected; SQSG_ERR_CAPACITY when its footprint can never fit. */
sqsg_status sqsg_server_submit(sqsg_server* server, const sqsg_job* job, uint64_t* ticket);
/* Waits for a ticket (timeout_us < 0: forever; SQSG_ERR_TIMEOUT when not done in time). The run's
 * statistics carry the job latency in timings_ns[SQSG_TIMING_TOTAL] (submission to result). */
sqsg_status sqsg_server_wait(sqsg_server* server, uint64_t ticket, int64_t timeout_us, sqsg_run** run);
sqsg_status sqsg_server_stats(sqsg_server* server, sqsg_server_counters* stats);
/* Persistent-kernel launches still running. CTAs leave after a bounded number of empty polls of
 * their ring (about 5 ms), so this drops to 0 soon after the server runs out of work. */
sqsg_status sqsg_server_running(sqsg_server* server, uint32_t* launches);
sqsg_status sqsg_server_destroy(sqsg_server* server);

#ifdef __cplusplus
}
#endif

#endif /* SQSGEN_B200_H */
