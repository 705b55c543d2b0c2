// Context object behind the opaque fdp_ctx handle.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>

#include "../../include/oneesan_fdp.h"
#include "fdp_launch.h"

struct fdp_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::map<int, fdp::DevTables> tables;  // per frontier width
  uint32_t *d_main = nullptr;            // run_sync state, [M][lanes]
  uint32_t *d_blk = nullptr;             // run_sync state, [D][lanes]
  size_t cap_main = 0, cap_blk = 0;
  unsigned long long *d_acc = nullptr;   // first-row dot accumulators
  uint32_t *d_res = nullptr;             // residues on the device
  uint32_t *h_res = nullptr;             // residues, pinned host
  unsigned int *d_err = nullptr;         // run_sync pass error word (device)
  unsigned int *h_err = nullptr;         // its copy after the pass (pinned host)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // A second stream for the sweep of the second lane span (lanes 8..): the
  // spans touch disjoint panels, so their cell launches run as two chains.
  cudaStream_t span_stream = nullptr;
  cudaEvent_t span_fork = nullptr, span_join = nullptr;
  fdp::LaunchCfg cfg;
  std::mutex mu;         // serialises run_sync / apply_cells / time_cells / tuning
  std::mutex tables_mu;  // guards `tables` (also used by the serving thread)
  struct fdp_server *server = nullptr;  // request loop (fdp_server_start)
  ~fdp_ctx();
};

fdp_status fdp_ctx_tables(fdp_ctx *c, int W, const fdp::DevTables **out);
fdp_status fdp_ctx_tables_cap(fdp_ctx *c, int W, int cap, const fdp::DevTables **out);
fdp_status fdp_prepare_pass(fdp_ctx *c, int W, const fdp::DevTables **full);
// One residue pass of L lanes on stream s.  With span_stream (and fork /
// join events) given, a pass of more than 8 lanes sweeps its second lane span
// on that stream, concurrently with the first on s.
fdp_status fdp_enqueue_pass(fdp_ctx *c, const fdp::DevTables &t, int L, const uint32_t *mods, uint32_t *main,
                            uint32_t *blk, unsigned long long *acc, uint32_t *d_res, uint32_t *h_res,
                            unsigned int *d_err, cudaStream_t s, uint64_t *launches,
                            cudaStream_t span_stream = nullptr, cudaEvent_t fork = nullptr,
                            cudaEvent_t join = nullptr);
// A computation's error word: a kernel that gives up on a bounded wait writes
// a nonzero value to it.  Each computation (a run_sync graph, one problem of a
// run_multi_sync graph, one served request) owns its word in its own buffers;
// the reset is enqueued before its passes and the read-back after them, on the
// same stream, so concurrent computations never see each other's failures.
cudaError_t fdp_enqueue_err_reset(unsigned int *d_err, cudaStream_t s);
cudaError_t fdp_enqueue_err_read(unsigned int *h_err, const unsigned int *d_err, cudaStream_t s);
void fdp_set_last_error(const char *msg);
fdp_status fdp_cuda_status(cudaError_t e, const char *what);
void fdp_server_shutdown(fdp_ctx *c);
