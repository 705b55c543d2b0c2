// Host-side launchers for the frontier-DP kernels (dispatch on index width and
// on K = residues interleaved per state).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "fdp_item.cuh"

namespace fdp {

constexpr int kMaxLanes = 16;  // K = 1..16 residues interleaved per state
constexpr int kCarryItems = 16;  // default states per lane of a grouped chunk with carry-over queues

// Per-(width, height cap) device table blob.
struct DevTables {
  void *ptr = nullptr;
  bool u64 = false;
  int W = 0;
  int cap = 1000;  // FDP_FULL_CAP: the full space
};
cudaError_t upload_tables(int W, int cap, DevTables *out);
void free_tables(DevTables *t);

struct LaunchCfg {
  int block = 256;
  int grid = 0;              // 0: sized from occupancy (a multiple of the SM count)
  bool split_panels = false; // several panels: one single-panel launch per panel
  bool bounded_prefix = true;  // first rows in height-bounded spaces
  int lane_items = 8;        // items per lane of a warp chunk of the cell kernel
  int share_min = 4;         // share the chunk's prefix decode when it walks >= this many positions
  int compact_max_p = 7;     // cells p <= this update a chunk's items grouped by centre type (-1: never)
  int compact_items = 0;     // states per lane of a compacted chunk (without carry-over 1..FDP_REC_MAX_ITEMS;
                             // 0: 4 for one span, 2 when closure sources are staged, which leaves L1
                             // room; with carry-over 1..16, 0: kCarryItems)
  int compact_carry = 0;     // grouped cells queue heads across chunks so every update runs 32 items
                             // (1 on, -1 off, 0 automatic: on when the lanes fit one span)
  int row_init = 0;          // strip rows filled directly by the row-k initialiser (0: automatic, -1: never)
  bool row_init_tensor = true;  // the initialiser's products on the tensor cores (else the CUDA cores)
  int split_spans_min_p = 1;    // cells p >= this run each span of a several-span lane count as its own launch
  bool span_chains = true;  // with every cell split, each span's row sweeps run as a chain of launches of
                            // their own, concurrent with the other span's (n=22, 14 lanes: pass 17.20 -> 16.83 s)
};

template <typename Idx, int K>
cudaError_t launch_cell_t(const CellArgs &a, const LaunchCfg &cfg, cudaStream_t s);
template <typename Idx, int K>
cudaError_t launch_first_row_t(const FirstRowArgs &a, bool dot, cudaStream_t s);

// One cell p on [M][K] / [D][K] arrays: one kernel launch, or one per lane
// span or panel when the configuration splits them; *kernels (if given) is
// increased by the launches made.
cudaError_t launch_cell(const DevTables &t, int K, const uint32_t *mods, uint32_t *main, uint32_t *blk, int p,
                        bool blk_in_zero, bool blk_out_p1, const LaunchCfg &cfg, cudaStream_t s,
                        uint64_t *kernels = nullptr);
// main[rank(first-row state)] = 1 for every first-row mask.
cudaError_t launch_first_row_init(const DevTables &t, int K, uint32_t *main, cudaStream_t s);
// acc[k] += sum over first-row states of main[.][k]; then residues[k] = acc[k] mod p_k.
cudaError_t launch_first_row_dot(const DevTables &t, int K, const uint32_t *mods, const uint32_t *main,
                                 unsigned long long *acc, uint32_t *residues, cudaStream_t s);

// Every word of the K lanes of the first N states set to 1 (row 0 in the
// height-1 space: every such word is a first-row state with coefficient 1).
cudaError_t launch_fill_ones(uint32_t *a, uint64_t words, cudaStream_t s);
// Move a K-lane state vector, in place, from the space `from` to the larger
// space `to` of the same width (ranks only grow), staging through `tmp`
// (tmp_words words, not overlapping `a`); words of `to` outside the image are
// zeroed.
cudaError_t enqueue_expand(const DevTables &from, const DevTables &to, int K, uint32_t *a, uint32_t *tmp,
                           uint64_t tmp_words, cudaStream_t s, uint64_t *launches = nullptr);

// Upload (once per device) the count tables enqueue_expand uses for these caps;
// must run outside stream capture.
cudaError_t prepare_expand_tables(const std::vector<int> &caps);

// Operator-surface helpers.
cudaError_t launch_rank_words(int width, const uint64_t *words, uint64_t *ranks, uint64_t count, cudaStream_t s);
cudaError_t launch_unrank_words(int width, const uint64_t *ranks, uint64_t *words, uint64_t count, cudaStream_t s);
cudaError_t launch_ternary_index(const uint32_t *codes, uint32_t *index, uint64_t count, cudaStream_t s);
cudaError_t launch_ternary_index_chunked(int chunk, const uint32_t *codes, uint32_t *index, uint64_t count,
                                         cudaStream_t s);

int device_sm_count();

}  // namespace fdp
