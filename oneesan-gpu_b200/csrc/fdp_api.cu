// C ABI of the frontier-DP engine (include/oneesan_fdp.h).
#include <atomic>
#include <chrono>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/oneesan_fdp.h"
#include "fdp_api_internal.h"
#include "fdp_host.h"
#include "fdp_launch.h"
#include "fdp_rowinit_dev.h"

using fdp::DevTables;

static thread_local std::string g_last_error;

#define FDP_RUN_MAX_MODULI 64

static fdp_status cuda_status(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return FDP_OK;
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();  // clear a sticky-free error so the context stays usable
  return e == cudaErrorMemoryAllocation ? FDP_ERR_HBM : FDP_ERR_CUDA;
}

#define FDP_CK(expr, what)                                  \
  do {                                                      \
    fdp_status _s = cuda_status((expr), (what));            \
    if (_s != FDP_OK) return _s;                            \
  } while (0)

extern "C" const char *fdp_version(void) { return "oneesan-fdp-b200 0.1 (sm_100a)"; }
extern "C" const char *fdp_last_error(void) { return g_last_error.c_str(); }

extern "C" uint64_t fdp_main_states(int width) { return fdp::main_states(width); }
extern "C" uint64_t fdp_blocked_states(int width) { return fdp::blocked_states(width); }
extern "C" uint64_t fdp_cell_bytes(int width, int p) {
  if (width < 2 || width > FDP_MAXW || p < 1 || p >= width) return 0;
  return fdp::cell_bytes(width, p);
}

static fdp_status check_problem(const fdp_problem *pr) {
  if (!pr || pr->n < 1 || pr->n > FDP_MAX_N || pr->k < 1 || !pr->moduli) {
    g_last_error = "problem: need 1 <= n <= 27, k >= 1 and a moduli array";
    return FDP_ERR_ARGS;
  }
  if (pr->lanes < 1 || pr->lanes > FDP_MAX_LANES) {
    g_last_error = "problem: lanes must be in 1..16";
    return FDP_ERR_ARGS;
  }
  for (int i = 0; i < pr->k; ++i)
    if (pr->moduli[i] < 2) {
      g_last_error = "problem: modulus must be in [2, 2^32-1]";
      return FDP_ERR_MODULUS;
    }
  return FDP_OK;
}

static int fit_row_init(int W, int R, bool bounded, int *cap);

extern "C" fdp_status fdp_plan(const fdp_problem *pr, uint64_t budget, fdp_plan_out *out) {
  fdp_status s = check_problem(pr);
  if (s != FDP_OK) return s;
  if (!out) return FDP_ERR_ARGS;
  const int W = pr->n + 1;
  const int lanes = pr->lanes < pr->k ? pr->lanes : pr->k;
  fdp_plan_out o{};
  o.n = pr->n;
  o.width = W;
  o.k = pr->k;
  o.lanes = lanes;
  o.passes = (pr->k + lanes - 1) / lanes;
  o.index_bits = fdp::needs_u64(W) ? 64 : 32;
  o.main_states = fdp::main_states(W);
  o.blocked_states = fdp::blocked_states(W);
  o.state_bytes = 4ull * (o.main_states + o.blocked_states) * uint64_t(lanes);
  o.scratch_bytes = 0;
  o.table_bytes = o.index_bits == 64 ? sizeof(fdp::WidthTables<uint64_t>) : sizeof(fdp::WidthTables<uint32_t>);
  o.total_bytes = o.state_bytes + o.table_bytes + (1u << 20);
  o.rows = fdp::sweep_rows(W);
  o.cells_per_row = W - 1;
  // Rows run in height-bounded spaces first (fdp_set_tuning bounded_prefix),
  // then in the full space.
  // The first init_rows - 1 sweep rows are replaced by the row-k initialiser
  // (default tuning, when its scratch fits).
  std::vector<int> caps;
  if (W >= 4) caps = fdp::bounded_prefix_caps(W);
  int R = fdp::auto_row_init_rows(W), rcap = 0;
  if (R >= 2) R = fit_row_init(W, R, true, &rcap);
  o.init_rows = R;
  const int first_row = R >= 2 ? R : 1;
  o.bounded_rows = 0;
  o.alg_bytes_per_residue = 0;
  o.transitions_per_residue = 0;
  for (int row = first_row; row <= o.rows; ++row) {
    const int cap = row <= int(caps.size()) ? caps[size_t(row - 1)] : FDP_FULL_CAP;
    if (cap < FDP_FULL_CAP) ++o.bounded_rows;
    o.alg_bytes_per_residue += fdp::row_bytes(W, cap);
    o.transitions_per_residue += uint64_t(o.cells_per_row) * fdp::cell_transitions(W, cap);
  }
  // Width tables a pass uploads: the full space, each bounded space and the
  // height-1 space of row 0; the expansion tables fit in the 1 MiB margin.
  const uint64_t ntables = 1 + (caps.empty() ? 0 : caps.size() + 1);
  o.sweep_peak_bytes = o.state_bytes + ntables * o.table_bytes + (1u << 20);
  o.init_peak_bytes = o.sweep_peak_bytes + (R >= 2 ? fdp::row_init_tables(W, R, rcap) : 0);
  o.total_bytes = o.init_peak_bytes > o.sweep_peak_bytes ? o.init_peak_bytes : o.sweep_peak_bytes;
  o.fits = o.total_bytes <= budget ? 1 : 0;
  *out = o;
  return FDP_OK;
}

extern "C" fdp_status fdp_create(fdp_ctx **out, int device) {
  if (!out) return FDP_ERR_ARGS;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) {
    cudaGetLastError();
    g_last_error = "no CUDA device visible";
    return FDP_ERR_GPU_COUNT;
  }
  if (device < 0 || device >= count) {
    g_last_error = "device index out of range";
    return FDP_ERR_GPU_COUNT;
  }
  FDP_CK(cudaSetDevice(device), "cudaSetDevice");
  auto *c = new fdp_ctx();
  c->device = device;
  fdp_status s = cuda_status(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream");
  if (s == FDP_OK) s = cuda_status(cudaMalloc(&c->d_acc, sizeof(unsigned long long) * FDP_MAX_LANES), "acc");
  if (s == FDP_OK) s = cuda_status(cudaMalloc(&c->d_res, sizeof(uint32_t) * FDP_MAX_LANES), "res");
  if (s == FDP_OK) s = cuda_status(cudaMallocHost(&c->h_res, sizeof(uint32_t) * FDP_RUN_MAX_MODULI), "pinned res");
  if (s == FDP_OK) s = cuda_status(cudaMalloc(&c->d_err, sizeof(unsigned int)), "error word");
  if (s == FDP_OK) s = cuda_status(cudaMallocHost(&c->h_err, sizeof(unsigned int)), "pinned error word");
  if (s == FDP_OK) s = cuda_status(cudaEventCreate(&c->ev0), "event");
  if (s == FDP_OK) s = cuda_status(cudaEventCreate(&c->ev1), "event");
  if (s == FDP_OK) s = cuda_status(cudaStreamCreateWithFlags(&c->span_stream, cudaStreamNonBlocking), "span stream");
  if (s == FDP_OK) s = cuda_status(cudaEventCreateWithFlags(&c->span_fork, cudaEventDisableTiming), "span event");
  if (s == FDP_OK) s = cuda_status(cudaEventCreateWithFlags(&c->span_join, cudaEventDisableTiming), "span event");
  if (s != FDP_OK) {
    fdp_destroy(c);
    return s;
  }
  *out = c;
  return FDP_OK;
}

fdp_ctx::~fdp_ctx() {
  fdp_server_shutdown(this);
  cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  for (auto &kv : tables) fdp::free_tables(&kv.second);
  if (d_main) cudaFree(d_main);
  if (d_blk) cudaFree(d_blk);
  if (d_acc) cudaFree(d_acc);
  if (d_res) cudaFree(d_res);
  if (h_res) cudaFreeHost(h_res);
  if (d_err) cudaFree(d_err);
  if (h_err) cudaFreeHost(h_err);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (span_fork) cudaEventDestroy(span_fork);
  if (span_join) cudaEventDestroy(span_join);
  if (span_stream) cudaStreamDestroy(span_stream);
  if (stream) cudaStreamDestroy(stream);
}

extern "C" void fdp_destroy(fdp_ctx *ctx) { delete ctx; }

fdp_status fdp_ctx_tables_cap(fdp_ctx *c, int W, int cap, const DevTables **out) {
  std::lock_guard<std::mutex> lk(c->tables_mu);
  const int key = W * 4096 + (cap >= FDP_FULL_CAP ? 4095 : cap);
  auto it = c->tables.find(key);
  if (it == c->tables.end()) {
    DevTables t;
    FDP_CK(fdp::upload_tables(W, cap, &t), "upload tables");
    it = c->tables.emplace(key, t).first;
  }
  *out = &it->second;
  return FDP_OK;
}

fdp_status fdp_ctx_tables(fdp_ctx *c, int W, const DevTables **out) {
  return fdp_ctx_tables_cap(c, W, FDP_FULL_CAP, out);
}

// Strip rows R the row-k initialiser fills directly for width W (0: the pass
// starts from row 0), and the height cap of the space row R runs in.  Used
// when the fill's scratch fits the blocked buffer (D words per lane, dead
// before the first sweep).
// The largest strip of at most R rows whose fill fits the blocked buffer.
static int fit_row_init(int W, int R, bool bounded, int *cap) {
  if (R > W - 1) R = W - 1;  // the state after row R-1 <= the last sweep row
  if (R > 7) R = 7;
  const std::vector<int> caps = (bounded && W >= 4) ? fdp::bounded_prefix_caps(W) : std::vector<int>{};
  for (; R >= 2; --R) {
    *cap = R <= int(caps.size()) ? caps[size_t(R - 1)] : FDP_FULL_CAP;
    if (fdp::row_init_scratch(W, R, *cap) <= fdp::blocked_states(W)) return R;
  }
  return 0;
}

static int row_init_rows(const fdp_ctx *c, int W, int *cap) {
  int R = c->cfg.row_init;
  if (R == 0) R = fdp::auto_row_init_rows(W);
  if (R < 2) return 0;
  return fit_row_init(W, R, c->cfg.bounded_prefix, cap);
}

// Every device table a residue pass of width W reads, uploaded before any
// stream capture starts (allocation and blocking copies cannot be captured).
fdp_status fdp_prepare_pass(fdp_ctx *c, int W, const DevTables **full) {
  fdp_status s = fdp_ctx_tables(c, W, full);
  if (s != FDP_OK) return s;
  int rcap = 0;
  if (const int R = row_init_rows(c, W, &rcap)) FDP_CK(fdp::prepare_row_init(W, R, rcap), "row-k initialiser tables");
  if (!c->cfg.bounded_prefix || W < 4) return s;
  std::vector<int> caps = fdp::bounded_prefix_caps(W);
  caps.push_back(1);
  const DevTables *t = nullptr;
  for (int cap : caps)
    if ((s = fdp_ctx_tables_cap(c, W, cap, &t)) != FDP_OK) return s;
  caps.push_back(FDP_FULL_CAP);
  FDP_CK(fdp::prepare_expand_tables(caps), "expand tables");
  return FDP_OK;
}

static fdp_status ensure_buffer(uint32_t **buf, size_t *cap, size_t bytes, const char *what) {
  if (*cap >= bytes && *buf) return FDP_OK;
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *cap = 0;
  FDP_CK(cudaMalloc(buf, bytes ? bytes : 4), what);
  *cap = bytes;
  return FDP_OK;
}

// Enqueue one whole residue pass on `s`: the row-0 state, the row sweeps, the
// first-row dot product and the residue copy to pinned host memory.  With the
// bounded prefix (c->cfg.bounded_prefix) row 0 is the height-1 space with every
// coefficient 1 and row r runs in the space of height cap r + 1 while that
// space is small; the state grows in place between them (the blocked buffer,
// dead at row boundaries, stages the move).  `blk` must hold D x L words of
// the full space.
// Test hook: the next `count` error-word resets write a nonzero value, as if
// a kernel had given up on a bounded wait (fdp_test_inject_pass_errors).
static std::atomic<int> g_injected_errors{0};

cudaError_t fdp_enqueue_err_reset(unsigned int *d_err, cudaStream_t s) {
  int v = g_injected_errors.load();
  while (v > 0 && !g_injected_errors.compare_exchange_weak(v, v - 1)) {
  }
  return cudaMemsetAsync(d_err, v > 0 ? 1 : 0, sizeof(unsigned int), s);
}

cudaError_t fdp_enqueue_err_read(unsigned int *h_err, const unsigned int *d_err, cudaStream_t s) {
  return cudaMemcpyAsync(h_err, d_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, s);
}

extern "C" fdp_status fdp_test_inject_pass_errors(int count) {
  if (count < 0) return FDP_ERR_ARGS;
  g_injected_errors.store(count);
  return FDP_OK;
}

fdp_status fdp_enqueue_pass(fdp_ctx *c, const DevTables &t, int L, const uint32_t *mods, uint32_t *main,
                            uint32_t *blk, unsigned long long *acc, uint32_t *d_res, uint32_t *h_res,
                            unsigned int *d_err, cudaStream_t s, uint64_t *launches, cudaStream_t span_stream,
                            cudaEvent_t fork, cudaEvent_t join) {
  const int W = t.W;
  const uint64_t M = fdp::main_states(W), D = fdp::blocked_states(W);
  uint64_t n = 0;
  fdp_status st = FDP_OK;
  // Rows 1..B run in height-bounded spaces (caps[r-1] for row r), the rest in
  // the full space.
  const std::vector<int> caps = (c->cfg.bounded_prefix && W >= 4) ? fdp::bounded_prefix_caps(W) : std::vector<int>{};
  const int B = int(caps.size());
  auto space = [&](int cap, const DevTables **out) -> fdp_status {
    if (cap >= FDP_FULL_CAP) {
      *out = &t;
      return FDP_OK;
    }
    return fdp_ctx_tables_cap(c, W, cap, out);
  };
  const DevTables *prev = nullptr;
  int next_row = 1;
  int rcap = 0;
  if (const int R = row_init_rows(c, W, &rcap)) {
    // Rows 0..R-1 at once: the state after row R-1, filled into row R's space
    // (the blocked buffer is the fill's scratch).
    if ((st = space(rcap, &prev)) != FDP_OK) return st;
    FDP_CK(fdp::enqueue_row_init(W, R, rcap, L, mods, main, blk, D * uint64_t(L), c->cfg.row_init_tensor, d_err, s,
                                 &n),
           "row-k initialiser");
    next_row = R;
  } else if (B > 0) {
    // Row 0 in the height-1 space: every word is a first-row state, coefficient 1.
    if ((st = space(1, &prev)) != FDP_OK) return st;
    FDP_CK(fdp::launch_fill_ones(main, fdp::main_states_capped(W, 1) * uint64_t(L), s), "row-0 fill");
    ++n;
  } else {
    FDP_CK(cudaMemsetAsync(main, 0, size_t(M) * L * 4, s), "zero main");
    FDP_CK(fdp::launch_first_row_init(t, L, main, s), "row-0 init");
    prev = &t;
    ++n;
  }
  for (int row = next_row; row <= B && row <= fdp::sweep_rows(W); ++row) {
    const DevTables *cur = nullptr;
    if ((st = space(caps[size_t(row - 1)], &cur)) != FDP_OK) return st;
    if (cur != prev) FDP_CK(fdp::enqueue_expand(*prev, *cur, L, main, blk, D * uint64_t(L), s, &n), "grow state");
    for (int p = W - 1; p >= 1; --p) {
      FDP_CK(fdp::launch_cell(*cur, L, mods, main, blk, p, p == W - 1, false, c->cfg, s, &n), "bounded cell");
    }
    prev = cur;
  }
  if (prev != &t) FDP_CK(fdp::enqueue_expand(*prev, t, L, main, blk, D * uint64_t(L), s, &n), "grow state");
  const int row0 = next_row > B + 1 ? next_row : B + 1;
  const bool chains = span_stream && fork && join && c->cfg.span_chains && L > 8 && !c->cfg.split_panels &&
                      c->cfg.split_spans_min_p <= 1 && row0 <= fdp::sweep_rows(W);
  if (chains) {
    // Each lane span is laid out as a lane count of its own at its first
    // panel's offset and no cell reads another span's panels, so the spans'
    // row sweeps run as two chains of launches, joined before the read-out.
    FDP_CK(cudaEventRecord(fork, s), "span fork");
    FDP_CK(cudaStreamWaitEvent(span_stream, fork, 0), "span fork");
    for (int l0 = 0, i = 0; l0 < L; ++i) {
      const int le = fdp::span_end_of(L, l0);
      cudaStream_t ss = i == 0 ? s : span_stream;
      for (int row = row0; row <= fdp::sweep_rows(W); ++row)
        for (int p = W - 1; p >= 1; --p)
          FDP_CK(fdp::launch_cell(t, le - l0, mods + l0, main + size_t(l0) * M, blk + size_t(l0) * D, p, p == W - 1,
                                  false, c->cfg, ss, &n),
                 "cell");
      l0 = le;
    }
    FDP_CK(cudaEventRecord(join, span_stream), "span join");
    FDP_CK(cudaStreamWaitEvent(s, join, 0), "span join");
  } else {
    for (int row = row0; row <= fdp::sweep_rows(W); ++row)
      for (int p = W - 1; p >= 1; --p) {
        FDP_CK(fdp::launch_cell(t, L, mods, main, blk, p, p == W - 1, false, c->cfg, s, &n), "cell");
      }
  }
  FDP_CK(fdp::launch_first_row_dot(t, L, mods, main, acc, d_res, s), "first-row dot");
  n += 2;
  if (h_res) FDP_CK(cudaMemcpyAsync(h_res, d_res, sizeof(uint32_t) * L, cudaMemcpyDeviceToHost, s), "residue copy");
  if (launches) *launches += n;
  return FDP_OK;
}

extern "C" fdp_status fdp_run_sync(fdp_ctx *c, const fdp_problem *pr, uint32_t *residues_out, fdp_run_stats *st) {
  if (!c || !residues_out) return FDP_ERR_ARGS;
  fdp_status s = check_problem(pr);
  if (s != FDP_OK) return s;
  if (pr->k > FDP_RUN_MAX_MODULI) {
    g_last_error = "run_sync: at most 64 moduli per call";
    return FDP_ERR_ARGS;
  }
  std::lock_guard<std::mutex> lk(c->mu);
  auto t0 = std::chrono::steady_clock::now();
  FDP_CK(cudaSetDevice(c->device), "cudaSetDevice");
  const int W = pr->n + 1;
  const DevTables *t = nullptr;
  if ((s = fdp_prepare_pass(c, W, &t)) != FDP_OK) return s;
  const int lanes = pr->lanes < pr->k ? pr->lanes : pr->k;
  const uint64_t M = fdp::main_states(W), D = fdp::blocked_states(W);
  if ((s = ensure_buffer(&c->d_main, &c->cap_main, size_t(M) * lanes * 4, "main state")) != FDP_OK) return s;
  if ((s = ensure_buffer(&c->d_blk, &c->cap_blk, size_t(D) * lanes * 4, "blocked state")) != FDP_OK) return s;
  // Every pass (lanes residues each) is captured into ONE graph, run with one launch.
  fdp_run_stats acc{};
  auto c0 = std::chrono::steady_clock::now();
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  FDP_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  uint64_t launches = 0;
  fdp_status es = cuda_status(fdp_enqueue_err_reset(c->d_err, c->stream), "error word");
  for (int done = 0; done < pr->k && es == FDP_OK; done += lanes) {
    const int L = (pr->k - done) < lanes ? (pr->k - done) : lanes;
    es = fdp_enqueue_pass(c, *t, L, pr->moduli + done, c->d_main, c->d_blk, c->d_acc, c->d_res, c->h_res + done,
                          c->d_err, c->stream, &launches, c->span_stream, c->span_fork, c->span_join);
  }
  if (es == FDP_OK) es = cuda_status(fdp_enqueue_err_read(c->h_err, c->d_err, c->stream), "error word");
  cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
  if (es != FDP_OK) {
    if (g) cudaGraphDestroy(g);
    return es;
  }
  FDP_CK(ce, "end capture");
  ce = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  FDP_CK(ce, "graph instantiate");
  acc.capture_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
  cudaEventRecord(c->ev0, c->stream);
  ce = cudaGraphLaunch(ge, c->stream);
  cudaEventRecord(c->ev1, c->stream);
  cudaError_t se = cudaStreamSynchronize(c->stream);
  cudaGraphExecDestroy(ge);
  FDP_CK(ce, "graph launch");
  FDP_CK(se, "residue pass");
  if (*c->h_err) {
    g_last_error = "residue pass: a bounded wait on the device gave up; the residues are invalid";
    return FDP_ERR_CUDA;
  }
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  acc.device_s = ms * 1e-3;
  acc.kernel_launches = launches;
  for (int i = 0; i < pr->k; ++i) residues_out[i] = c->h_res[i];
  fdp_plan_out po{};
  fdp_plan(pr, ~0ull, &po);
  acc.alg_bytes = po.alg_bytes_per_residue * uint64_t(pr->k);
  acc.transitions = po.transitions_per_residue * uint64_t(pr->k);
  acc.wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (st) *st = acc;
  return FDP_OK;
}

extern "C" fdp_status fdp_apply_cells(fdp_ctx *c, int width, int p_hi, int p_lo, int lanes, const uint32_t *moduli,
                                      uint32_t *d_main, uint32_t *d_block, void *stream) {
  // Checked first, before anything that needs a context or a device.
  if (!fdp::panel_aligned(lanes, d_main) || !fdp::panel_aligned(lanes, d_block)) {
    g_last_error = "apply_cells: d_main and d_block must be aligned to one word of the widest lane panel "
                   "(32 bytes for 8 or more lanes, 16 for 4-7, 8 for 2-3)";
    return FDP_ERR_ARGS;
  }
  if (!c || !moduli || !d_main || !d_block) return FDP_ERR_ARGS;
  if (width < 2 || width > FDP_MAXW || p_lo < 1 || p_hi >= width || p_lo > p_hi || lanes < 1 ||
      lanes > FDP_MAX_LANES) {
    g_last_error = "apply_cells: need 2 <= width <= 28, 1 <= p_lo <= p_hi < width, 1 <= lanes <= 16";
    return FDP_ERR_ARGS;
  }
  for (int i = 0; i < lanes; ++i)
    if (moduli[i] < 2) return FDP_ERR_MODULUS;
  std::lock_guard<std::mutex> lk(c->mu);
  FDP_CK(cudaSetDevice(c->device), "cudaSetDevice");
  const DevTables *t = nullptr;
  fdp_status s = fdp_ctx_tables(c, width, &t);
  if (s != FDP_OK) return s;
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  for (int p = p_hi; p >= p_lo; --p)
    FDP_CK(fdp::launch_cell(*t, lanes, moduli, d_main, d_block, p, false, true, c->cfg, st), "cell");
  return FDP_OK;
}

extern "C" fdp_status fdp_rank_words(fdp_ctx *c, int width, const uint64_t *d_words, uint64_t *d_ranks,
                                     uint64_t count, void *stream) {
  if (!c || width < 1 || width > FDP_MAXW || (count && (!d_words || !d_ranks))) return FDP_ERR_ARGS;
  FDP_CK(cudaSetDevice(c->device), "cudaSetDevice");
  FDP_CK(fdp::launch_rank_words(width, d_words, d_ranks, count, stream ? (cudaStream_t)stream : c->stream), "rank");
  return FDP_OK;
}

extern "C" fdp_status fdp_unrank_words(fdp_ctx *c, int width, const uint64_t *d_ranks, uint64_t *d_words,
                                       uint64_t count, void *stream) {
  if (!c || width < 1 || width > FDP_MAXW || (count && (!d_words || !d_ranks))) return FDP_ERR_ARGS;
  FDP_CK(cudaSetDevice(c->device), "cudaSetDevice");
  FDP_CK(fdp::launch_unrank_words(width, d_ranks, d_words, count, stream ? (cudaStream_t)stream : c->stream),
         "unrank");
  return FDP_OK;
}

extern "C" fdp_status fdp_ternary_index(fdp_ctx *c, const uint32_t *d_codes, uint32_t *d_index, uint64_t count,
                                        void *stream) {
  if (!c || (count && (!d_codes || !d_index))) return FDP_ERR_ARGS;
  FDP_CK(cudaSetDevice(c->device), "cudaSetDevice");
  FDP_CK(fdp::launch_ternary_index(d_codes, d_index, count, stream ? (cudaStream_t)stream : c->stream), "ternary");
  return FDP_OK;
}

extern "C" fdp_status fdp_ternary_index_chunked(fdp_ctx *c, int chunk, const uint32_t *d_codes, uint32_t *d_index,
                                                uint64_t count, void *stream) {
  if (!c || (chunk != 4 && chunk != 7) || (count && (!d_codes || !d_index))) {
    g_last_error = "ternary_index_chunked: chunk must be 4 or 7";
    return FDP_ERR_ARGS;
  }
  FDP_CK(cudaSetDevice(c->device), "cudaSetDevice");
  FDP_CK(fdp::launch_ternary_index_chunked(chunk, d_codes, d_index, count, stream ? (cudaStream_t)stream : c->stream),
         "ternary chunked");
  return FDP_OK;
}

extern "C" fdp_status fdp_time_cells(fdp_ctx *c, const fdp_problem *pr, int rows, double *cell_ms) {
  if (!c || !cell_ms || rows < 1) return FDP_ERR_ARGS;
  fdp_status s = check_problem(pr);
  if (s != FDP_OK) return s;
  std::lock_guard<std::mutex> lk(c->mu);
  FDP_CK(cudaSetDevice(c->device), "cudaSetDevice");
  const int W = pr->n + 1;
  if (W < 3) return FDP_ERR_ARGS;
  const DevTables *t = nullptr;
  if ((s = fdp_ctx_tables(c, W, &t)) != FDP_OK) return s;
  const int L = pr->lanes < pr->k ? pr->lanes : pr->k;
  const uint64_t M = fdp::main_states(W), D = fdp::blocked_states(W);
  if ((s = ensure_buffer(&c->d_main, &c->cap_main, size_t(M) * L * 4, "main state")) != FDP_OK) return s;
  if ((s = ensure_buffer(&c->d_blk, &c->cap_blk, size_t(D) * L * 4, "blocked state")) != FDP_OK) return s;
  std::vector<cudaEvent_t> ev(size_t(rows) * W * 2);
  for (auto &e : ev) FDP_CK(cudaEventCreate(&e), "event");
  // One untimed launch first: the first launch of a kernel variant also loads
  // its module and sets its shared-memory limit.
  fdp_status rs = cuda_status(
      fdp::launch_cell(*t, L, pr->moduli, c->d_main, c->d_blk, W - 1, true, false, c->cfg, c->stream), "cell");
  for (int r = 0; r < rows && rs == FDP_OK; ++r)
    for (int p = W - 1; p >= 1 && rs == FDP_OK; --p) {
      cudaEventRecord(ev[(size_t(r) * W + p) * 2], c->stream);
      rs = cuda_status(fdp::launch_cell(*t, L, pr->moduli, c->d_main, c->d_blk, p, p == W - 1, false, c->cfg,
                                        c->stream), "cell");
      cudaEventRecord(ev[(size_t(r) * W + p) * 2 + 1], c->stream);
    }
  cudaError_t se = cudaStreamSynchronize(c->stream);
  if (rs == FDP_OK) rs = cuda_status(se, "timed cells");
  if (rs == FDP_OK) {
    for (int p = 0; p < W; ++p) cell_ms[p] = 0;
    for (int r = 0; r < rows; ++r)
      for (int p = W - 1; p >= 1; --p) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev[(size_t(r) * W + p) * 2], ev[(size_t(r) * W + p) * 2 + 1]);
        cell_ms[p] += ms / rows;
      }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  return rs;
}

fdp_status fdp_cuda_status(cudaError_t e, const char *what) { return cuda_status(e, what); }

// Lets other translation units of the library report a message through
// fdp_last_error().
void fdp_set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

extern "C" fdp_status fdp_set_tuning(fdp_ctx *c, const fdp_tuning *t) {
  if (!c || !t) return FDP_ERR_ARGS;
  if (t->block < 64 || t->block > 256 || t->block % 32 || t->grid < 0 || t->lane_items < 0 || t->lane_items > 64 ||
      t->share_min < 0 || t->compact_max_p < -1 || t->compact_carry < -1 || t->compact_carry > 1 ||
      t->compact_items < 0 || t->compact_items > (t->compact_carry < 0 ? FDP_REC_MAX_ITEMS : 16) ||
      t->row_init_rows < -1 || t->row_init_rows > 7 || t->row_init_product < 0 || t->row_init_product > 1 ||
      t->split_spans_min_p < 0) {
    g_last_error =
        "tuning: block must be a multiple of 32 in 64..256, grid >= 0, lane_items 0..64, share_min >= 0, "
        "compact_max_p >= -1, compact_carry -1..1, compact_items 0..16 (0..4 with compact_carry -1; "
        "a value above 4 is used only where heads carry over), "
        "row_init_rows -1..7, row_init_product 0..1";
    return FDP_ERR_ARGS;
  }
  std::lock_guard<std::mutex> lk(c->mu);
  c->cfg.block = t->block;
  c->cfg.grid = t->grid;
  c->cfg.split_panels = t->split_panels != 0;
  c->cfg.bounded_prefix = t->bounded_prefix != 0;
  c->cfg.lane_items = t->lane_items > 0 ? t->lane_items : fdp::LaunchCfg{}.lane_items;
  c->cfg.share_min = t->share_min > 0 ? t->share_min : fdp::LaunchCfg{}.share_min;
  c->cfg.compact_max_p = t->compact_max_p != 0 ? t->compact_max_p : fdp::LaunchCfg{}.compact_max_p;
  c->cfg.compact_items = t->compact_items;
  c->cfg.compact_carry = t->compact_carry;
  c->cfg.row_init = t->row_init_rows;
  c->cfg.row_init_tensor = t->row_init_product == 0;
  c->cfg.split_spans_min_p = t->split_spans_min_p > 0 ? t->split_spans_min_p : fdp::LaunchCfg{}.split_spans_min_p;
  return FDP_OK;
}

extern "C" fdp_status fdp_get_tuning(fdp_ctx *c, fdp_tuning *t) {
  if (!c || !t) return FDP_ERR_ARGS;
  std::lock_guard<std::mutex> lk(c->mu);
  t->block = c->cfg.block;
  t->grid = c->cfg.grid;
  t->split_panels = c->cfg.split_panels ? 1 : 0;
  t->bounded_prefix = c->cfg.bounded_prefix ? 1 : 0;
  t->lane_items = c->cfg.lane_items;
  t->share_min = c->cfg.share_min;
  t->compact_max_p = c->cfg.compact_max_p;
  t->compact_items = c->cfg.compact_items;
  t->compact_carry = c->cfg.compact_carry;
  t->row_init_rows = c->cfg.row_init;
  t->row_init_product = c->cfg.row_init_tensor ? 0 : 1;
  t->split_spans_min_p = c->cfg.split_spans_min_p;
  return FDP_OK;
}

// One problem of fdp_run_multi_sync: its buffers and its forked stream.
struct MultiPart {
  const DevTables *t = nullptr;
  int lanes = 1;
  uint32_t *main = nullptr, *blk = nullptr, *res = nullptr;
  unsigned long long *acc = nullptr;
  unsigned int *err = nullptr;  // this problem's error word
  cudaStream_t s = nullptr;
  cudaEvent_t done = nullptr;
  cudaStream_t span_s = nullptr;  // the second lane span's sweep
  cudaEvent_t span_fork = nullptr, span_join = nullptr;
};

extern "C" fdp_status fdp_run_multi_sync(fdp_ctx *c, const fdp_problem *probs, int count, uint32_t *residues_out,
                                         fdp_run_stats *st) {
  if (!c || !probs || count < 1 || count > 64 || !residues_out) return FDP_ERR_ARGS;
  int total_k = 0;
  for (int i = 0; i < count; ++i) {
    fdp_status s = check_problem(&probs[i]);
    if (s != FDP_OK) return s;
    total_k += probs[i].k;
  }
  std::lock_guard<std::mutex> lk(c->mu);
  auto t0 = std::chrono::steady_clock::now();
  FDP_CK(cudaSetDevice(c->device), "cudaSetDevice");
  std::vector<MultiPart> parts(static_cast<size_t>(count));
  uint32_t *pinned = nullptr;
  cudaEvent_t fork = nullptr;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  fdp_status rs = FDP_OK;
  uint64_t launches = 0;
  auto cleanup = [&]() {
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    for (size_t i = 0; i < parts.size(); ++i) {
      MultiPart &p = parts[i];
      if (p.main) cudaFree(p.main);
      if (p.blk) cudaFree(p.blk);
      if (p.acc) cudaFree(p.acc);
      if (p.res) cudaFree(p.res);
      if (p.err) cudaFree(p.err);
      if (p.s) cudaStreamDestroy(p.s);
      if (p.done) cudaEventDestroy(p.done);
      if (p.span_s) cudaStreamDestroy(p.span_s);
      if (p.span_fork) cudaEventDestroy(p.span_fork);
      if (p.span_join) cudaEventDestroy(p.span_join);
    }
    if (pinned) cudaFreeHost(pinned);
    if (fork) cudaEventDestroy(fork);
  };
#define MULTI_CK(expr, what)                   \
  do {                                         \
    rs = cuda_status((expr), (what));          \
    if (rs != FDP_OK) { cleanup(); return rs; } \
  } while (0)
  // Residues of every problem, then one error word per problem.
  MULTI_CK(cudaMallocHost(&pinned, sizeof(uint32_t) * size_t(total_k + count)), "pinned residues");
  MULTI_CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event");
  for (int i = 0; i < count; ++i) {
    MultiPart &p = parts[size_t(i)];
    const int W = probs[i].n + 1;
    if ((rs = fdp_prepare_pass(c, W, &p.t)) != FDP_OK) { cleanup(); return rs; }
    p.lanes = probs[i].lanes < probs[i].k ? probs[i].lanes : probs[i].k;
    MULTI_CK(cudaMalloc(&p.main, size_t(fdp::main_states(W)) * p.lanes * 4), "multi main state");
    MULTI_CK(cudaMalloc(&p.blk, size_t(fdp::blocked_states(W)) * p.lanes * 4 + 4), "multi blocked state");
    MULTI_CK(cudaMalloc(&p.acc, sizeof(unsigned long long) * FDP_MAX_LANES), "multi acc");
    MULTI_CK(cudaMalloc(&p.res, sizeof(uint32_t) * FDP_MAX_LANES), "multi res");
    MULTI_CK(cudaMalloc(&p.err, sizeof(unsigned int)), "multi error word");
    MULTI_CK(cudaStreamCreateWithFlags(&p.s, cudaStreamNonBlocking), "multi stream");
    MULTI_CK(cudaEventCreateWithFlags(&p.done, cudaEventDisableTiming), "multi event");
    if (p.lanes > 8) {
      MULTI_CK(cudaStreamCreateWithFlags(&p.span_s, cudaStreamNonBlocking), "multi stream");
      MULTI_CK(cudaEventCreateWithFlags(&p.span_fork, cudaEventDisableTiming), "multi event");
      MULTI_CK(cudaEventCreateWithFlags(&p.span_join, cudaEventDisableTiming), "multi event");
    }
  }
  auto c0 = std::chrono::steady_clock::now();
  MULTI_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaEventRecord(fork, c->stream);
  int off = 0;
  for (int i = 0; i < count && rs == FDP_OK; ++i) {
    MultiPart &p = parts[size_t(i)];
    cudaStreamWaitEvent(p.s, fork, 0);
    rs = cuda_status(fdp_enqueue_err_reset(p.err, p.s), "error word");
    for (int done = 0; done < probs[i].k && rs == FDP_OK; done += p.lanes) {
      const int L = (probs[i].k - done) < p.lanes ? (probs[i].k - done) : p.lanes;
      rs = fdp_enqueue_pass(c, *p.t, L, probs[i].moduli + done, p.main, p.blk, p.acc, p.res, pinned + off + done,
                            p.err, p.s, &launches, p.span_s, p.span_fork, p.span_join);
    }
    if (rs == FDP_OK)
      rs = cuda_status(fdp_enqueue_err_read(reinterpret_cast<unsigned int *>(pinned + total_k + i), p.err, p.s),
                       "error word");
    cudaEventRecord(p.done, p.s);
    cudaStreamWaitEvent(c->stream, p.done, 0);
    off += probs[i].k;
  }
  cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
  if (rs != FDP_OK) { cleanup(); return rs; }
  MULTI_CK(ce, "end capture");
  MULTI_CK(cudaGraphInstantiate(&ge, g, 0), "graph instantiate");
  const double cap_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
  cudaEventRecord(c->ev0, c->stream);
  MULTI_CK(cudaGraphLaunch(ge, c->stream), "graph launch");
  cudaEventRecord(c->ev1, c->stream);
  MULTI_CK(cudaStreamSynchronize(c->stream), "multi pass");
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  for (int i = 0; i < count; ++i)
    if (pinned[total_k + i]) {
      g_last_error = "multi pass: a bounded wait on the device gave up in problem " + std::to_string(i) +
                     "; the residues are invalid";
      cleanup();
      return FDP_ERR_CUDA;
    }
  for (int i = 0; i < total_k; ++i) residues_out[i] = pinned[i];
  if (st) {
    fdp_run_stats acc{};
    acc.device_s = ms * 1e-3;
    acc.capture_s = cap_s;
    acc.kernel_launches = launches;
    for (int i = 0; i < count; ++i) {
      fdp_plan_out po{};
      fdp_plan(&probs[i], ~0ull, &po);
      acc.alg_bytes += po.alg_bytes_per_residue * uint64_t(probs[i].k);
      acc.transitions += po.transitions_per_residue * uint64_t(probs[i].k);
    }
    acc.wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *st = acc;
  }
  cleanup();
  return FDP_OK;
#undef MULTI_CK
}
