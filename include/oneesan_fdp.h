/*
 * oneesan_fdp.h -- C ABI of the B200 frontier (transfer-matrix) DP engine.
 *
 * Counts simple corner-to-corner paths on an (n+1)x(n+1) vertex grid as uint32
 * residues modulo primes below 2^32 (README.md:3 of the reference).  Every
 * entry point takes plain pointers and sizes; device pointers are CUDA device
 * addresses on the context's device, host pointers are ordinary memory.
 *
 * The reference's own boundary is a process (solver binary argv + one stdout
 * line per modulus, GB.cu:2090-2101 and GB.cu:2257, with
 * GB.cu = src/cuda/b300/oneesan_cuda_gridfp_b300_hbm32_factorized_fullprerank_orbit_blockfused_groupbatch_batch.cu).
 * The CLI in this repository (oneesan_solver) keeps that contract and is
 * itself a client of the functions below.  Each declaration names the
 * reference interface it replaces.
 *
 * Conventions
 *   - Status codes are returned, never exits or exceptions.  Codes 1-5 and 34
 *     equal the reference solver's exit codes for the same condition
 *     (GB.cu:2098-2184).
 *   - One context per device; calls on one context are serialised by the
 *     caller, except fdp_submit / fdp_poll, which are thread-safe.
 *   - Residues are canonical in [0, p); moduli are in [2, 2^32 - 1].
 *   - Coefficient vectors are in canonical rank order (GB.cu:1568 rank_full).
 *     The `lanes` residues of a state (one per modulus) are stored in panels:
 *     lanes are grouped greedily 8, 4, 2, 1 at a time (lanes = 14 -> panels
 *     {0-7}, {8-11}, {12-13}); the panel whose first lane is L0 and whose
 *     width is PW is an array [N][PW] that starts at word L0 * N, where N is
 *     the number of states of the vector.  For lanes = 1, 2, 4 or 8 this is
 *     the plain interleaved layout word[state * lanes + l].
 */
#ifndef ONEESAN_FDP_H
#define ONEESAN_FDP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fdp_status {
  FDP_OK = 0,
  FDP_ERR_ARGS = 1,         /* bad arguments (reference exit 1)                       */
  FDP_ERR_GPU_COUNT = 2,    /* no usable GPU (reference exit 2)                       */
  FDP_ERR_WINDOW = 4,       /* request does not fit the scratch/lanes limit (exit 4)  */
  FDP_ERR_HBM = 5,          /* HBM budget or device memory exhausted (exit 5)         */
  FDP_ERR_CUDA = 6,         /* a CUDA runtime error; see fdp_last_error()             */
  FDP_ERR_MODULUS = 34,     /* modulus outside [2, 2^32-1] (reference exit 34 class)  */
  FDP_PENDING = 100,        /* fdp_poll: request not finished yet                     */
  FDP_TIMEOUT = 101,        /* a bounded wait ran out                                  */
  FDP_ERR_NOT_FOUND = 102   /* unknown request slot                                    */
} fdp_status;

#define FDP_MAX_N 27      /* widest grid: W = n+1 <= 28 (GB.cu:28 MAXW)        */
#define FDP_MAX_LANES 16  /* residues interleaved per state in one pass         */

typedef struct fdp_ctx fdp_ctx;

/* A problem: one grid size and a set of moduli. */
typedef struct fdp_problem {
  int n;                    /* grid cells per side, 1..27                         */
  int k;                    /* number of moduli                                    */
  const uint32_t *moduli;   /* k moduli (host memory)                              */
  int lanes;                /* residues per pass: 1 = plain, k = batched (<=16)   */
} fdp_problem;

/* Memory and work plan of a problem (GRIDFP_PLAN_ONLY output, GB.cu:2117-2168). */
typedef struct fdp_plan_out {
  int n, width, k, lanes, passes;
  int index_bits;                   /* 32 or 64                                   */
  uint64_t main_states;             /* H_DP[W][1]                                 */
  uint64_t blocked_states;          /* H_DP[W-1][1]                               */
  uint64_t state_bytes;             /* 4 (M + D) lanes: the whole device footprint */
  uint64_t scratch_bytes;           /* 0: the transition is in place              */
  uint64_t table_bytes;             /* per-width index tables                     */
  uint64_t total_bytes;
  int rows;                         /* row sweeps per residue                     */
  int bounded_rows;                 /* of which in height-bounded spaces (prefix) */
  int init_rows;                    /* rows of vertices filled by the row-k initialiser (default tuning) */
  int cells_per_row;                /* W - 1                                      */
  uint64_t alg_bytes_per_residue;   /* sum over cells of fdp_cell_bytes            */
  uint64_t transitions_per_residue; /* sum over cells of (M + D)                  */
  int fits;                         /* total_bytes <= budget                      */
  uint64_t sweep_peak_bytes;        /* device bytes held during the row sweeps:
                                       state, every width table of the pass
                                       (bounded spaces included), small buffers
                                       (the PLAN line's dp_peak_gib)            */
  uint64_t init_peak_bytes;         /* device bytes held while the row-k
                                       initialiser fills the state: the above
                                       plus its tables; its scratch is the
                                       blocked state (the PLAN line's
                                       row6_peak_gib)                           */
} fdp_plan_out;

/* Per-call timing (the reference reports wall_s and phase sums, GB.cu:2257). */
typedef struct fdp_run_stats {
  double wall_s;          /* host wall clock of the whole call                   */
  double device_s;        /* CUDA-event time of the captured sweep(s)             */
  double capture_s;       /* graph capture + instantiate                          */
  uint64_t kernel_launches;
  uint64_t alg_bytes;     /* algorithmic bytes moved (all residues)               */
  uint64_t transitions;   /* frontier transitions (all residues)                  */
} fdp_run_stats;

/* Library version string. */
const char *fdp_version(void);
/* Message of the last failing CUDA call on this thread ("" if none). */
const char *fdp_last_error(void);

/*
 * Pure host planner, no device access.  Replaces GRIDFP_PLAN_ONLY=1
 * (GB.cu:2117-2168) and the HBM admission check (GB.cu:2182-2186).
 */
fdp_status fdp_plan(const fdp_problem *problem, uint64_t hbm_budget_bytes, fdp_plan_out *out);

/* Context on one device (replaces DeviceCtx::init and the allocations, GB.cu:2172-2186). */
fdp_status fdp_create(fdp_ctx **out, int device);
void fdp_destroy(fdp_ctx *ctx);

/*
 * Residues of the path count for every modulus of `problem` (k <= 64),
 * synchronously.  The k moduli run in passes of `lanes` residues per state;
 * all passes are captured into one CUDA graph and run with one launch.
 * lanes = 1 is the plain one-modulus-per-launch-sequence form (the
 * reference's residue loop, GB.cu:2211-2258); lanes = k is one batched pass.
 * residues_out has k entries.
 */
fdp_status fdp_run_sync(fdp_ctx *ctx, const fdp_problem *problem, uint32_t *residues_out, fdp_run_stats *stats);

/*
 * Several problems (grid sizes and moduli sets) in ONE captured CUDA graph:
 * each problem's passes are captured on its own forked stream, joined at the
 * end, and the graph runs with a single launch, so the problems overlap on the
 * GPU.  residues_out receives the residues of problem 0, then problem 1, ...
 * (sum of k entries).  stats covers the whole graph.  No counterpart in the
 * reference, which runs one n per binary (the batched form of this engine).
 */
fdp_status fdp_run_multi_sync(fdp_ctx *ctx, const fdp_problem *problems, int count, uint32_t *residues_out,
                              fdp_run_stats *stats);

/*
 * Operator level: apply cells p_hi, p_hi-1, ..., p_lo of one row sweep to
 * caller-owned device vectors (width = n+1, main: lanes x M words, block:
 * lanes x D words, both in the panel layout above).
 * The blocked input is consumed at p_hi; the blocked output of p_lo is left in
 * `block` (all zero when p_lo = 1).  Replaces process_window_batched_io for a
 * window (GB.cu:1701-1742) as exercised by tests/groupbatch_operator_test.cu,
 * and the reverse (pull) sweep kernels (R2.cu:1039-1155, R2.cu =
 * src/cuda/b300/oneesan_cuda_gridfp_b300_hbm32_factorized_reverse2_row6crt20_batch.cu):
 * this engine's cell operator is itself a pull sweep.  With all lane moduli
 * equal, the lanes are independent vectors under one modulus, the GROUPBATCH
 * lane semantics (src/cuda/b300/groupbatch_interleaved.cuh).
 * `stream` is a cudaStream_t (0 = the context's stream); the call is async.
 * `main` and `block` must be aligned to one word of the widest panel: 32
 * bytes for 8 or more lanes (an 8-lane word is one 256-bit access), 16 for
 * 4-7, 8 for 2-3 (cudaMalloc gives 256); otherwise FDP_ERR_ARGS.
 */
fdp_status fdp_apply_cells(fdp_ctx *ctx, int width, int p_hi, int p_lo, int lanes, const uint32_t *moduli,
                           uint32_t *d_main, uint32_t *d_block, void *stream);

/*
 * Profiling: run `rows` row sweeps of the problem's first pass (its first
 * `lanes` moduli) on the context's resident state, each cell a separate launch
 * bracketed by CUDA events on the context's stream, and return the mean
 * duration of every cell p in cell_ms[p] (cell_ms has `width` entries, index
 * 0 unused).  Values in the state are irrelevant to the timing: the kernel's
 * access pattern depends only on indices.  Replaces the CUDA-event phase
 * timers of GRIDFP_PROFILE_BATCH=1 (src/cuda/b300/factor_transfer_batch.cuh:110-158).
 */
fdp_status fdp_time_cells(fdp_ctx *ctx, const fdp_problem *problem, int rows, double *cell_ms);

/*
 * Launch tuning of the cell kernel for this context (what the autotuner sets;
 * the reference's GRIDFP_THREADS and scheduling knobs, GB.cu:2190,
 * scripts/run/autotune.py:157-300).  block: threads per CTA (64..256, a
 * multiple of 32); grid: CTAs per launch (0 = sized from occupancy, a multiple
 * of the SM count); split_panels: for lane counts that need several panels,
 * run one launch per panel instead of one launch that stages closure sources
 * in shared memory; bounded_prefix: run row r in the space of words of height
 * <= r + 1 while that space is much smaller than the full one (the reference's
 * bounded-height prefix, GB.cu:1825-1838: row r never reaches a higher height),
 * growing the state in place between rows.  lane_items: each warp of the cell
 * kernel takes chunks of 32 * lane_items consecutive blocked states (0 = the
 * default, 8); share_min: when a cell's high prefix is at least this many
 * symbols long, the symbols a whole chunk shares are decoded once per chunk
 * (0 = the default, 4; a value above the width never shares); compact_max_p:
 * cells p <= compact_max_p, where the items of one warp mix centre types,
 * decode a chunk's items first and update them grouped by type (0 = the
 * default, 7; -1 = never); compact_items: states per lane of such a cell's
 * chunks (0 = automatic: without carry-over 4 when the lanes fit one span of
 * 8, else 2, which leaves more of the SM's on-chip memory to L1); row_init_rows: the
 * pass starts from the state after the first row_init_rows rows of vertices,
 * computed directly by the row-k initialiser (a column automaton of that
 * strip, the reference's row-5/row-6 initialisers, GB.cu:874-1032) instead of
 * row sweeps, when its scratch fits the blocked state buffer (0 = automatic:
 * 7 rows from width 18 up, 6 from width 14; -1 = never); row_init_product:
 * the initialiser's products on the tensor cores (0, tcgen05 with 8-bit limbs)
 * or on the CUDA cores (1); split_spans_min_p: for lane counts above 8 (two
 * spans), cells p >= split_spans_min_p run each span as its own single-span
 * launch instead of one launch that stages closure sources (0 = the
 * default, 1: every cell; a value above the width never splits); compact_carry: the grouped cells keep the heads of one type that
 * do not fill a warp queued for the warp's next chunk, so every grouped
 * update runs on 32 items (1 = on, -1 = group each chunk alone, 0 = automatic:
 * on when the lanes fit one span of 8, the case where it was measured
 * faster); with carry-over compact_items may be 1..16 (0 = 16) and only sets
 * the chunk whose prefix decode is shared; without it values above 4 count
 * as 4.  Results never depend on these settings.
 */
typedef struct fdp_tuning {
  int block;
  int grid;
  int split_panels;
  int bounded_prefix;  /* first rows in height-bounded spaces (default 1)       */
  int lane_items;      /* states per lane of a warp chunk, 0..64 (0: default)   */
  int share_min;       /* shortest prefix decoded once per chunk (0: default)   */
  int compact_max_p;   /* highest cell grouped by centre type (0: default, -1: none) */
  int compact_items;   /* states per lane of a grouped chunk, 0..16 (0: automatic) */
  int row_init_rows;   /* rows filled by the row-k initialiser, 2..7 (0: automatic, -1: none) */
  int row_init_product; /* its products on the tensor cores (0, default) or CUDA cores (1) */
  int split_spans_min_p; /* cells p >= this run each lane span as its own launch (0: default) */
  int compact_carry;   /* grouped cells queue heads across chunks: 1 on, -1 off, 0 automatic */
} fdp_tuning;
fdp_status fdp_set_tuning(fdp_ctx *ctx, const fdp_tuning *tuning);
fdp_status fdp_get_tuning(fdp_ctx *ctx, fdp_tuning *tuning);

/*
 * Serving: a request loop with continuous batching.  No counterpart in the
 * reference, which runs one process per job (the served form of this engine).
 *
 * fdp_server_start reserves hbm_budget_bytes of device memory once and starts
 * a scheduler thread.  Requests (n, moduli) queue in arrival order; a request
 * is admitted as soon as one of max_active slots and enough of the reserved
 * pool are free (its frontier, 4 (M+D) lanes bytes, stays on the device until
 * it finishes).  Later, smaller requests may pass a request that does not fit
 * yet, unless it has waited longer than max_bypass_s.  Each admitted request
 * runs its residue pass(es) as one CUDA graph on its own stream, so admitted
 * requests overlap on the GPU and finish independently.  A request whose
 * moduli fill less than one pass of max_lanes takes along later queued
 * requests of the same n while their moduli fit, so one pass serves them all
 * (fdp_request_info then reports the shared pass's lanes).  Results are exact
 * and the same as fdp_run_sync's for the same problem.
 */
typedef struct fdp_server_config {
  uint64_t hbm_budget_bytes;  /* device pool reserved for frontiers              */
  int max_active;             /* concurrent requests on the GPU (1..64)          */
  int max_lanes;              /* residues per pass (1..16), shared by same-n riders */
  double max_bypass_s;        /* backfill limit; <= 0 means 30 s                  */
} fdp_server_config;

typedef struct fdp_request_info {
  double queue_s;      /* submit -> admitted                                     */
  double run_s;        /* admitted -> completion seen by the scheduler           */
  double latency_s;    /* submit -> completion                                   */
  double device_s;     /* CUDA-event time of the request's graph                 */
  int lanes, passes;
  uint64_t state_bytes;
} fdp_request_info;

typedef struct fdp_server_stats {
  uint64_t submitted, completed, failed, queued, running;
  uint64_t pool_bytes, bytes_in_use, peak_bytes_in_use;
  int peak_running;
} fdp_server_stats;

fdp_status fdp_server_start(fdp_ctx *ctx, const fdp_server_config *config);
/* Stops admitting, fails queued requests, waits for running ones, frees the pool. */
fdp_status fdp_server_stop(fdp_ctx *ctx);
/* Queue a request (problem->lanes is ignored; max_lanes applies).  Thread-safe.
 * FDP_ERR_HBM if it can never fit the pool. */
fdp_status fdp_submit(fdp_ctx *ctx, const fdp_problem *problem, uint64_t *request_id);
/* FDP_PENDING while queued or running; FDP_OK copies k residues, fills info
 * and forgets the request; an error status for a failed request.  Thread-safe. */
fdp_status fdp_poll(fdp_ctx *ctx, uint64_t request_id, uint32_t *residues_out, fdp_request_info *info);
/* fdp_poll with a bounded wait: FDP_TIMEOUT after timeout_ms. */
fdp_status fdp_wait(fdp_ctx *ctx, uint64_t request_id, int timeout_ms, uint32_t *residues_out,
                    fdp_request_info *info);
fdp_status fdp_server_get_stats(fdp_ctx *ctx, fdp_server_stats *stats);

/*
 * Autotuner (the reference's scripts/run/autotune.py:157-300 discipline:
 * admission from the memory plan, then one warm-up and `repeats` timed samples
 * per candidate, median, and a known-residue check that aborts on a wrong
 * answer).  Candidates: residues per pass (how the k moduli of the problem
 * split into passes; problem->lanes is the largest allowed), one launch vs one
 * launch per lane panel, and the CTA size; then, for the winner, the cell
 * kernel's scheduling knobs one at a time (lane_items, share_min,
 * compact_max_p, compact_carry, compact_items, and split_spans_min_p above 8 lanes; a change
 * is kept when the row is at least 0.5 % faster).  Each sample is a timed row sweep of the problem's own n on
 * the context's state buffers; the score is the estimated device seconds per
 * residue.  The known-answer check runs the tuned configuration at the
 * problem's own n when the reference publishes a residue mod 4294967291 for
 * it (n = 9, 18, 20, 21, 22, 23), else at n = 9.  The winner is applied to the context
 * (fdp_set_tuning) and returned; json_out (if not NULL) receives every
 * candidate record as a JSON document of at most json_cap bytes.
 */
typedef struct fdp_autotune_result {
  int lanes;                /* residues per pass                                  */
  int passes;               /* passes for the problem's k moduli                  */
  fdp_tuning tuning;        /* block / grid / split_panels                        */
  double row_ms;            /* median row-sweep time of the winner                */
  double s_per_residue;     /* estimated device seconds per residue              */
  double residues_per_hour; /* 3600 / s_per_residue                               */
  int candidates, rejected_memory;
  int check_n;              /* grid size of the known-residue check            */
} fdp_autotune_result;
fdp_status fdp_autotune(fdp_ctx *ctx, const fdp_problem *problem, uint64_t hbm_budget_bytes, int repeats,
                        fdp_autotune_result *out, char *json_out, size_t json_cap);

/*
 * Factorized transfer map: the cell operator (or two consecutive cells when
 * `paired`) as a CSR matrix of predecessor indices over the index space
 * [0, M) main + [M, M+D) blocked of one width, built on the device (count,
 * scan, fill, and a check that the fill pass agrees with the count pass) and
 * applied out of place: out_main = in_main + T x, out_block = T x.  Replaces
 * factor_transfer::{counts,fill,verify,apply}_kernel
 * (src/cuda/b300/factor_transfer_map.cuh:40-68) and its batched apply
 * (factor_transfer_batch.cuh:13-47); lanes follow the panel layout.
 * Widths whose M + D exceeds 2^32 are rejected (32-bit columns).
 */
typedef struct fdp_transfer_map fdp_transfer_map;
fdp_status fdp_transfer_map_build(fdp_ctx *ctx, int width, int p, int paired, fdp_transfer_map **out);
fdp_status fdp_transfer_map_info(const fdp_transfer_map *map, uint64_t *rows, uint64_t *edges,
                                 uint64_t *device_bytes);
fdp_status fdp_transfer_map_apply(fdp_ctx *ctx, const fdp_transfer_map *map, int lanes, const uint32_t *moduli,
                                  const uint32_t *d_in_main, const uint32_t *d_in_block, uint32_t *d_out_main,
                                  uint32_t *d_out_block, void *stream);
void fdp_transfer_map_destroy(fdp_transfer_map *map);

/*
 * Factorized transfer map over occupancy groups: one CSR per group shape,
 * reused for every conjugate group (the reference's
 * src/cuda/b300/factor_transfer_map.cuh:1-68 with its batched apply,
 * factor_transfer_batch.cuh:13-164).  A group is the set of words (main and
 * blocked) whose bottom `fixed` positions hold R or L exactly at the set bits
 * of a mask and N elsewhere; cell p (and p-1 when `paired`) leaves those
 * positions alone and its closures only swap R and L, so every group is closed
 * under the operator, and two groups with the same number `occupied` of set
 * bits are conjugate: moving the occupied symbols in order between the
 * positions keeps the canonical order and every source.  The CSR is built on
 * the device over the local ranks of the representative group (the bottom
 * `occupied` positions set) with the count / scan / fill / check sequence of
 * fdp_transfer_map_build; requires fixed <= p - 1 (p - 2 when paired) and
 * fixed <= 24.  fdp_factor_map_apply runs it on `groups` (<= max_groups <= 32)
 * groups at once for one modulus: the groups' values are gathered from the
 * global vectors (plain layout, one residue per state) into an arena with the
 * groups interleaved as columns, the CSR is applied column by column with one
 * reduction per output, and the results are scattered to their global ranks
 * in the output vectors (out_main = in_main + T x, out_block = T x on the
 * groups' rows; other rows are not written).  masks is host memory, each with
 * `occupied` set bits below bit `fixed`.  phase_ms (3 entries, may be NULL)
 * receives the CUDA-event times of gather, apply and scatter, the reference's
 * GRIDFP_PROFILE_BATCH phase timers (factor_transfer_batch.cuh:110-158); with
 * it the call waits for the stream.
 */
typedef struct fdp_factor_map fdp_factor_map;
fdp_status fdp_factor_map_build(fdp_ctx *ctx, int width, int p, int paired, int fixed, int occupied,
                                int max_groups, fdp_factor_map **out);
fdp_status fdp_factor_map_info(const fdp_factor_map *map, uint64_t *group_main, uint64_t *group_blocked,
                               uint64_t *edges, uint64_t *device_bytes);
fdp_status fdp_factor_map_apply(fdp_ctx *ctx, const fdp_factor_map *map, uint32_t modulus, int groups,
                                const uint32_t *masks, const uint32_t *d_in_main, const uint32_t *d_in_block,
                                uint32_t *d_out_main, uint32_t *d_out_block, void *stream, double *phase_ms);
void fdp_factor_map_destroy(fdp_factor_map *map);

/*
 * Two consecutive cells p, p-1 fused by recursive pull, out of place, without
 * storing the intermediate vector or a matrix (the reverse2 kernels,
 * R2.cu:1116-1155).  Same result as fdp_apply_cells(p, p-1).
 */
fdp_status fdp_reverse2_apply(fdp_ctx *ctx, int width, int p, int lanes, const uint32_t *moduli,
                              const uint32_t *d_in_main, const uint32_t *d_in_block, uint32_t *d_out_main,
                              uint32_t *d_out_block, void *stream);

/*
 * Residue read-out that allocates no device memory.  No counterpart in the
 * reference, whose solver owns all device memory itself.
 *
 * For callers that cannot let a library call cudaMalloc: a serving process or
 * framework whose own pool allocator already holds the GPU's memory (an
 * allocation would fail or break the pool's budget), or code that must not
 * take the device synchronisation cudaMalloc / cudaFree can cause.  Such a
 * caller runs the row sweeps on its own buffers (fdp_apply_cells) and then
 * reads the residues of its final state `d_main` (width x lanes, panel
 * layout) into `d_residues` (lanes uint32 in device memory) with this call;
 * `moduli` is host memory.  The dot product's 64-bit accumulators live in a
 * fixed array inside the library (128 bytes, 16 lanes), so widths above 28
 * or more than 16 lanes are rejected with FDP_ERR_ARGS.  The first call on a
 * device, with that device current, looks the array's device address up and
 * keeps it; make that first call before any stream capture, and do not call
 * this entry point again after destroying the device's primary context
 * (cudaDeviceReset).  Every call on a device shares the array; each call
 * clears it on `stream` first, but calls that overlap on the GPU race on it
 * and must be serialised.  `d_main` has the alignment fdp_apply_cells asks
 * of it (32 bytes for 8 or more lanes), or the call returns FDP_ERR_ARGS.
 */
fdp_status fdp_first_row_dot_noalloc(int width, int lanes, const uint32_t *moduli, const uint32_t *d_main,
                                     uint32_t *d_residues, void *stream);

/*
 * Fault injection for tests: the next `count` computations (a run_sync or
 * run_multi_sync problem, a served request) start with their device error
 * word already set, exactly as when one of their kernels gives up on a bounded
 * wait, so that each entry point's failure report can be checked without
 * making a kernel fail.  No counterpart in the reference.
 */
fdp_status fdp_test_inject_pass_errors(int count);

/* Canonical rank / unrank of frontier words on the device (GB.cu:1568 rank_full). */
fdp_status fdp_rank_words(fdp_ctx *ctx, int width, const uint64_t *d_words, uint64_t *d_ranks, uint64_t count,
                          void *stream);
fdp_status fdp_unrank_words(fdp_ctx *ctx, int width, const uint64_t *d_ranks, uint64_t *d_words, uint64_t count,
                            void *stream);

/* Ternary rank index on the device (src/common/ternary_rank_index.hpp:6-15). */
fdp_status fdp_ternary_index(fdp_ctx *ctx, const uint32_t *d_codes, uint32_t *d_index, uint64_t count, void *stream);
/*
 * The same index through a table of every code of `chunk` symbols (chunk 4 or
 * 7; 4^chunk entries): one table read per chunk of the code, the chunked
 * device conversion of the reference (GRIDFP_TRIT_CHUNK, R2.cu:23-55, tested
 * by tests/ternary_rank_index_test.cpp:7-27).  Codes of up to 16 symbols.
 */
fdp_status fdp_ternary_index_chunked(fdp_ctx *ctx, int chunk, const uint32_t *d_codes, uint32_t *d_index,
                                     uint64_t count, void *stream);

/*
 * Host helpers: state counts and the per-cell algorithmic byte model, the
 * minimum traffic of one cell of the in-place sweep for one modulus:
 * 4 x (every main word + the blocked input unless p = width-1)
 * + 4 x (main words that can change + the blocked output unless p = 1).
 */
uint64_t fdp_main_states(int width);
uint64_t fdp_blocked_states(int width);
uint64_t fdp_cell_bytes(int width, int p);

#ifdef __cplusplus
}
#endif
#endif /* ONEESAN_FDP_H */
