// Operator-surface variants of the per-cell transition: the factorized
// transfer map (CSR of predecessor indices, the reference's
// src/cuda/b300/factor_transfer_map.cuh:7-68 and factor_transfer_batch.cuh)
// and the two-cell pull ("reverse2", R2.cu:1116-1155 of the reference), both
// out of place over the full canonical space of one width.
//
// Index space: rows [0, M) are main targets, rows [M, M+D) blocked targets.
// For cell p the sources of a target are enumerated on words, restating the
// transition (src/common/gridfp_transition.hpp:113-146) in pull form:
//   main t:    t itself; LR <- NN, NR <- RN, NL <- LN (p >= 2); at p = 1 also
//              RN <- NR, LN <- NL and NN <- every RR closure (a depth-1 R above
//              flipped to L); plus the blocked word with position p removed
//              when t has N at p.
//   blocked b (p >= 2), centre c = b[p-1], u = b with N inserted at p:
//              c = R or L: u;  c = N: u with pair RL (if the height above is
//              >= 1), every LL closure (a depth-1 L below flipped to R) and
//              every RR closure (a depth-1 R above flipped to L).
// A paired step (p, p-1) composes the two: the sources at p of every source
// at p-1, with multiplicity.  The identity edge of a main row is implicit in
// the CSR (the first source of a main row is always the row itself).
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/oneesan_fdp.h"
#include "fdp_api_internal.h"
#include "fdp_host.h"
#include "fdp_launch.h"

namespace {

using ull = unsigned long long;

struct Counts {
  ull H[FDP_MAXW + 1][FDP_HT];
};

__device__ __forceinline__ uint32_t get(uint64_t w, int k) { return uint32_t(w >> (2 * k)) & 3u; }
__device__ __forceinline__ uint64_t put(uint64_t w, int k, uint32_t v) {
  return (w & ~(3ull << (2 * k))) | (uint64_t(v) << (2 * k));
}
__device__ __forceinline__ uint64_t put_pair(uint64_t w, int p, uint32_t hi, uint32_t lo) {
  return put(put(w, p, hi), p - 1, lo);
}
__device__ __forceinline__ uint64_t drop_at(uint64_t w, int k) {  // remove position k
  const uint64_t low = (1ull << (2 * k)) - 1;
  return ((w & ~low) >> 2) | (w & low);
}
__device__ __forceinline__ uint64_t insert_at(uint64_t w, int k, uint32_t v) {  // insert v at position k
  const uint64_t low = k ? ((1ull << (2 * k)) - 1) : 0;
  return (w & low) | (uint64_t(v) << (2 * k)) | ((w & ~low) << 2);
}

__device__ ull rank_word_dev(uint64_t m, int W, const ull (*H)[FDP_HT]) {
  ull r = 0;
  int h = 1;
  for (int pos = W - 1; pos >= 0; --pos) {
    const uint32_t s = get(m, pos);
    if (s > fdp::SYM_N) r += H[pos][h];
    if (s > fdp::SYM_R && h > 0) r += H[pos][h - 1];
    h += s == fdp::SYM_L ? 1 : (s == fdp::SYM_R ? -1 : 0);
  }
  return r;
}

__device__ uint64_t unrank_word_dev(ull r, int W, const ull (*H)[FDP_HT]) {
  uint64_t m = 0;
  int h = 1;
  for (int pos = W - 1; pos >= 0; --pos) {
    ull z = H[pos][h];
    if (r < z) continue;
    r -= z;
    z = h > 0 ? H[pos][h - 1] : 0ull;
    if (r < z) { m |= uint64_t(fdp::SYM_R) << (2 * pos); --h; continue; }
    r -= z;
    m |= uint64_t(fdp::SYM_L) << (2 * pos);
    ++h;
  }
  return m;
}

// Index spaces the sources are ranked in.  FullSpace: the canonical ranks of
// every word of a width.  GroupSpace: the local ranks of one occupancy group,
// the words whose bottom `fixed` positions carry R/L exactly at the set bits
// of `occ` (N elsewhere); H holds the counts of that constrained space, so
// the canonical order restricted to the group numbers it 0, 1, ...  Both
// widths (main W, blocked W-1) share the constraint: it is on absolute
// positions below every position a cell touches.
struct FullSpace {
  const ull (*H)[FDP_HT];
  __device__ ull rank(uint64_t w, int width) const { return rank_word_dev(w, width, H); }
  __device__ uint64_t unrank(ull r, int width) const { return unrank_word_dev(r, width, H); }
};

struct GroupSpace {
  const ull (*H)[FDP_HT];
  int fixed;
  uint32_t occ;
  __device__ bool n_ok(int q) const { return q >= fixed || !((occ >> q) & 1u); }
  __device__ bool rl_ok(int q) const { return q >= fixed || ((occ >> q) & 1u); }
  __device__ ull rank(uint64_t m, int width) const {
    ull r = 0;
    int h = 1;
    for (int pos = width - 1; pos >= 0; --pos) {
      const uint32_t s = get(m, pos);
      if (s > fdp::SYM_N && n_ok(pos)) r += H[pos][h];
      if (s > fdp::SYM_R && h > 0 && rl_ok(pos)) r += H[pos][h - 1];
      h += s == fdp::SYM_L ? 1 : (s == fdp::SYM_R ? -1 : 0);
    }
    return r;
  }
  __device__ uint64_t unrank(ull r, int width) const {
    uint64_t m = 0;
    int h = 1;
    for (int pos = width - 1; pos >= 0; --pos) {
      ull z = n_ok(pos) ? H[pos][h] : 0ull;
      if (r < z) continue;
      r -= z;
      z = (h > 0 && rl_ok(pos)) ? H[pos][h - 1] : 0ull;
      if (r < z) { m |= uint64_t(fdp::SYM_R) << (2 * pos); --h; continue; }
      r -= z;
      m |= uint64_t(fdp::SYM_L) << (2 * pos);
      ++h;
    }
    return m;
  }
};

// Height just above position p (after reading positions W-1..p+1 top-down).
__device__ int height_above(uint64_t w, int W, int p) {
  int h = 1;
  for (int q = W - 1; q > p; --q) {
    const uint32_t s = get(w, q);
    h += s == fdp::SYM_L ? 1 : (s == fdp::SYM_R ? -1 : 0);
  }
  return h;
}

// RR closures: every R at depth 1 scanning up from position p+1 of w (whose
// pair at (p, p-1) is NN), flipped to L, with the pair set to RR.
template <class Emit>
__device__ void rr_closures(uint64_t w, int W, int p, Emit &&emit) {
  int depth = 1;
  for (int q = p + 1; q < W && depth > 0; ++q) {
    const uint32_t s = get(w, q);
    if (s == fdp::SYM_R) {
      if (depth == 1) emit(put(put_pair(w, p, fdp::SYM_R, fdp::SYM_R), q, fdp::SYM_L));
      ++depth;
    } else if (s == fdp::SYM_L) {
      --depth;
    }
  }
}

// LL closures: every L at depth 1 scanning down from position p-2 of w (pair NN
// at (p, p-1)), flipped to R, with the pair set to LL.
template <class Emit>
__device__ void ll_closures(uint64_t w, int p, Emit &&emit) {
  int depth = 1;
  for (int q = p - 2; q >= 0 && depth > 0; --q) {
    const uint32_t s = get(w, q);
    if (s == fdp::SYM_L) {
      if (depth == 1) emit(put(put_pair(w, p, fdp::SYM_L, fdp::SYM_L), q, fdp::SYM_R));
      ++depth;
    } else if (s == fdp::SYM_R) {
      --depth;
    }
  }
}

// Sources (indices into [0, M+D) of the space) of row i at cell p; main rows
// emit i first.
template <class Space, class Emit>
__device__ void step_sources(ull i, ull M, int W, int p, const Space &sp, Emit &&emit) {
  if (i < M) {
    const uint64_t t = sp.unrank(i, W);
    emit(i);
    auto main_src = [&](uint64_t s) { emit(sp.rank(s, W)); };
    const uint32_t a = get(t, p), b = get(t, p - 1);
    using namespace fdp;
    if (a == SYM_L && b == SYM_R) main_src(put_pair(t, p, SYM_N, SYM_N));
    if (a == SYM_N && b == SYM_R) main_src(put_pair(t, p, SYM_R, SYM_N));
    if (a == SYM_N && b == SYM_L) main_src(put_pair(t, p, SYM_L, SYM_N));
    if (p == 1) {
      if (a == SYM_R && b == SYM_N) main_src(put_pair(t, p, SYM_N, SYM_R));
      if (a == SYM_L && b == SYM_N) main_src(put_pair(t, p, SYM_N, SYM_L));
      if (a == SYM_N && b == SYM_N) rr_closures(t, W, p, main_src);
    }
    if (a == SYM_N) emit(M + sp.rank(drop_at(t, p), W - 1));
    return;
  }
  if (p < 2) return;  // no blocked output at p = 1
  const uint64_t bw = sp.unrank(i - M, W - 1);
  const uint64_t u = insert_at(bw, p, fdp::SYM_N);
  const uint32_t c = get(bw, p - 1);
  auto main_src = [&](uint64_t s) { emit(sp.rank(s, W)); };
  if (c != fdp::SYM_N) {
    main_src(u);
    return;
  }
  if (height_above(u, W, p) >= 1) main_src(put_pair(u, p, fdp::SYM_R, fdp::SYM_L));
  ll_closures(u, p, main_src);
  rr_closures(u, W, p, main_src);
}

template <class Space, class Emit>
__device__ void sources(ull i, ull M, int W, int p, bool paired, const Space &sp, Emit &&emit) {
  if (!paired) {
    step_sources(i, M, W, p, sp, emit);
    return;
  }
  step_sources(i, M, W, p - 1, sp, [&](ull j) { step_sources(j, M, W, p, sp, emit); });
}

__device__ void load_counts(ull (*sH)[FDP_HT], const Counts *c) {
  for (int k = threadIdx.x; k < (FDP_MAXW + 1) * FDP_HT; k += blockDim.x) (&sH[0][0])[k] = (&c->H[0][0])[k];
  __syncthreads();
}

// The space of a CSR build: the full space (fixed = 0) or the occupancy group
// of `occ` on the bottom `fixed` positions, counts in shared memory.
struct SpaceArgs {
  const Counts *counts;
  int fixed;
  uint32_t occ;
};

template <bool Group>
struct SpaceOf;
template <>
struct SpaceOf<false> {
  using type = FullSpace;
  __device__ static FullSpace make(const ull (*sH)[FDP_HT], const SpaceArgs &) { return FullSpace{sH}; }
};
template <>
struct SpaceOf<true> {
  using type = GroupSpace;
  __device__ static GroupSpace make(const ull (*sH)[FDP_HT], const SpaceArgs &s) {
    return GroupSpace{sH, s.fixed, s.occ};
  }
};

template <bool Group>
__global__ void csr_count_kernel(SpaceArgs sa, ull M, ull total, int W, int p, bool paired, ull *rowlen) {
  __shared__ ull sH[FDP_MAXW + 1][FDP_HT];
  load_counts(sH, sa.counts);
  const auto sp = SpaceOf<Group>::make(sH, sa);
  for (ull i = ull(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += ull(gridDim.x) * blockDim.x) {
    ull n = 0;
    sources(i, M, W, p, paired, sp, [&](ull) { ++n; });
    rowlen[i] = n - (i < M ? 1 : 0);
  }
}

template <bool Group>
__global__ void csr_fill_kernel(SpaceArgs sa, ull M, ull total, int W, int p, bool paired, const ull *offsets,
                                uint32_t *columns, ull *errors) {
  __shared__ ull sH[FDP_MAXW + 1][FDP_HT];
  load_counts(sH, sa.counts);
  const auto sp = SpaceOf<Group>::make(sH, sa);
  ull bad = 0;
  for (ull i = ull(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += ull(gridDim.x) * blockDim.x) {
    ull pos = offsets[i];
    const ull end = offsets[i + 1];
    bool first = i < M;
    sources(i, M, W, p, paired, sp, [&](ull j) {
      if (first) {  // the identity edge stays implicit
        if (j != i) ++bad;
        first = false;
        return;
      }
      if (pos < end && j < total) columns[pos] = uint32_t(j);
      else ++bad;
      ++pos;
    });
    if (pos != end) ++bad;
  }
  if (bad) atomicAdd(errors, bad);
}

__device__ __forceinline__ size_t lane_addr(int K, ull N, ull s, int l) {
  int l0 = 0;
  while (true) {
    const int pw = (K - l0 >= 8) ? 8 : (K - l0 >= 4) ? 4 : (K - l0 >= 2) ? 2 : 1;
    if (l < l0 + pw) return size_t(l0) * N + size_t(s) * pw + (l - l0);
    l0 += pw;
  }
}

struct ApplyArgs {
  const uint32_t *in_main, *in_blk;
  uint32_t *out_main, *out_blk;
  ull M, D;
  int K;
  uint32_t mod[16];
};

__device__ __forceinline__ uint32_t src_value(const ApplyArgs &a, ull j, int l) {
  return j < a.M ? a.in_main[lane_addr(a.K, a.M, j, l)] : a.in_blk[lane_addr(a.K, a.D, j - a.M, l)];
}

__device__ __forceinline__ void store_row(const ApplyArgs &a, ull i, int l, ull sum) {
  const uint32_t v = uint32_t(sum % a.mod[l]);  // sum < 2^41: at most ~6W sources below 2^32
  if (i < a.M) a.out_main[lane_addr(a.K, a.M, i, l)] = v;
  else a.out_blk[lane_addr(a.K, a.D, i - a.M, l)] = v;
}

__global__ void csr_apply_kernel(ApplyArgs a, const ull *offsets, const uint32_t *columns) {
  const ull total = a.M + a.D;
  for (ull i = ull(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += ull(gridDim.x) * blockDim.x) {
    const ull b = offsets[i], e = offsets[i + 1];
    for (int l = 0; l < a.K; ++l) {
      ull sum = i < a.M ? a.in_main[lane_addr(a.K, a.M, i, l)] : 0ull;
      for (ull k = b; k < e; ++k) sum += src_value(a, columns[k], l);
      store_row(a, i, l, sum);
    }
  }
}

__global__ void reverse2_kernel(ApplyArgs a, const Counts *c, int W, int p) {
  __shared__ ull sH[FDP_MAXW + 1][FDP_HT];
  load_counts(sH, c);
  const FullSpace sp{sH};
  const ull total = a.M + a.D;
  for (ull i = ull(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += ull(gridDim.x) * blockDim.x) {
    ull sum[16];
    for (int l = 0; l < a.K; ++l) sum[l] = 0;
    sources(i, a.M, W, p, true, sp, [&](ull j) {
      if (j >= total) return;  // cannot happen for legal words; keeps every read in bounds
      for (int l = 0; l < a.K; ++l) sum[l] += src_value(a, j, l);
    });
    for (int l = 0; l < a.K; ++l) store_row(a, i, l, sum[l]);
  }
}

const Counts *device_counts() {
  static std::mutex mu;
  static std::vector<std::pair<int, Counts *>> per_dev;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  for (auto &pd : per_dev)
    if (pd.first == dev) return pd.second;
  Counts h;
  const fdp::CountTable &ct = fdp::counts();
  for (int w = 0; w <= FDP_MAXW; ++w)
    for (int k = 0; k < FDP_HT; ++k) h.H[w][k] = ct.H[w][k];
  Counts *d = nullptr;
  if (cudaMalloc(&d, sizeof(h)) != cudaSuccess) return nullptr;
  if (cudaMemcpy(d, &h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
  per_dev.push_back({dev, d});
  return d;
}

unsigned grid_for(ull n) {
  ull g = (n + 255) / 256, cap = ull(fdp::device_sm_count()) * 8;
  return unsigned(g < 1 ? 1 : (g > cap ? cap : g));
}

fdp_status check_apply(int width, int lanes, const uint32_t *moduli, const void *a, const void *b, const void *c,
                       const void *d) {
  if (width < 3 || width > FDP_MAXW || lanes < 1 || lanes > FDP_MAX_LANES || !moduli || !a || !b || !c || !d) {
    fdp_set_last_error("transfer: need 3 <= width <= 28, 1 <= lanes <= 16 and four device vectors");
    return FDP_ERR_ARGS;
  }
  if (fdp::main_states(width) + fdp::blocked_states(width) > 0xffffffffull) {
    fdp_set_last_error("transfer: width too large for 32-bit CSR columns");
    return FDP_ERR_ARGS;
  }
  for (int i = 0; i < lanes; ++i)
    if (moduli[i] < 2) return FDP_ERR_MODULUS;
  return FDP_OK;
}

}  // namespace

struct fdp_transfer_map {
  int device = 0, width = 0, p = 0, paired = 0;
  ull rows = 0, edges = 0;
  ull *offsets = nullptr;     // rows + 1
  uint32_t *columns = nullptr;
};

namespace {

// Count, scan, fill and check the CSR of one index space (rows [0, M) main,
// [M, total) blocked); the identity edge of main rows stays implicit.
template <bool Group>
fdp_status build_csr(fdp_ctx *c, const SpaceArgs &sa, ull M, ull total, int width, int p, bool paired,
                     ull **offsets_out, uint32_t **columns_out, ull *edges_out) {
  ull *offsets = nullptr, *err = nullptr;
  uint32_t *columns = nullptr;
  cudaError_t e;
  auto fail = [&](cudaError_t ce, const char *what) {
    if (err) cudaFree(err);
    if (offsets) cudaFree(offsets);
    if (columns) cudaFree(columns);
    return fdp_cuda_status(ce, what);
  };
  if ((e = cudaMalloc(&offsets, sizeof(ull) * (total + 1))) != cudaSuccess) return fail(e, "csr offsets");
  if ((e = cudaMalloc(&err, sizeof(ull))) != cudaSuccess) return fail(e, "csr errors");
  csr_count_kernel<Group><<<grid_for(total), 256, 0, c->stream>>>(sa, M, total, width, p, paired, offsets);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "csr count");
  std::vector<ull> off(total + 1);
  if ((e = cudaMemcpyAsync(off.data(), offsets, sizeof(ull) * total, cudaMemcpyDeviceToHost, c->stream)) !=
      cudaSuccess)
    return fail(e, "csr count copy");
  if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return fail(e, "csr count sync");
  ull run = 0;  // exclusive scan
  for (ull i = 0; i < total; ++i) {
    const ull len = off[i];
    off[i] = run;
    run += len;
  }
  off[total] = run;
  if ((e = cudaMemcpyAsync(offsets, off.data(), sizeof(ull) * (total + 1), cudaMemcpyHostToDevice, c->stream)) !=
      cudaSuccess)
    return fail(e, "csr offsets copy");
  if ((e = cudaMalloc(&columns, sizeof(uint32_t) * (run ? run : 1))) != cudaSuccess) return fail(e, "csr columns");
  if ((e = cudaMemsetAsync(err, 0, sizeof(ull), c->stream)) != cudaSuccess) return fail(e, "csr errors");
  csr_fill_kernel<Group><<<grid_for(total), 256, 0, c->stream>>>(sa, M, total, width, p, paired, offsets, columns,
                                                                 err);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "csr fill");
  ull bad = 0;
  if ((e = cudaMemcpyAsync(&bad, err, sizeof(ull), cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess)
    return fail(e, "csr verify copy");
  if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return fail(e, "csr fill sync");
  cudaFree(err);
  err = nullptr;
  if (bad) {
    fail(cudaSuccess, "");
    fdp_set_last_error("transfer map: the fill pass disagreed with the count pass");
    return FDP_ERR_CUDA;
  }
  *offsets_out = offsets;
  *columns_out = columns;
  *edges_out = run;
  return FDP_OK;
}

}  // namespace

extern "C" fdp_status fdp_transfer_map_build(fdp_ctx *c, int width, int p, int paired, fdp_transfer_map **out) {
  if (!c || !out || width < 3 || width > FDP_MAXW || p < 1 || p >= width || (paired && p < 2)) {
    fdp_set_last_error("transfer_map_build: need 3 <= width <= 28, 1 <= p < width (p >= 2 when paired)");
    return FDP_ERR_ARGS;
  }
  *out = nullptr;
  const ull M = fdp::main_states(width), D = fdp::blocked_states(width), total = M + D;
  if (total > 0xffffffffull) {
    fdp_set_last_error("transfer_map_build: width too large for 32-bit CSR columns");
    return FDP_ERR_ARGS;
  }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fdp_cuda_status(e, "cudaSetDevice");
  const Counts *cnt = device_counts();
  if (!cnt) return FDP_ERR_HBM;
  auto map = std::make_unique<fdp_transfer_map>();
  map->device = c->device;
  map->width = width;
  map->p = p;
  map->paired = paired ? 1 : 0;
  map->rows = total;
  const SpaceArgs sa{cnt, 0, 0u};
  fdp_status st = build_csr<false>(c, sa, M, total, width, p, paired != 0, &map->offsets, &map->columns, &map->edges);
  if (st != FDP_OK) return st;
  *out = map.release();
  return FDP_OK;
}

extern "C" fdp_status fdp_transfer_map_info(const fdp_transfer_map *m, uint64_t *rows, uint64_t *edges,
                                            uint64_t *device_bytes) {
  if (!m) return FDP_ERR_ARGS;
  if (rows) *rows = m->rows;
  if (edges) *edges = m->edges;
  if (device_bytes) *device_bytes = sizeof(ull) * (m->rows + 1) + sizeof(uint32_t) * m->edges;
  return FDP_OK;
}

extern "C" void fdp_transfer_map_destroy(fdp_transfer_map *m) {
  if (!m) return;
  cudaSetDevice(m->device);
  if (m->offsets) cudaFree(m->offsets);
  if (m->columns) cudaFree(m->columns);
  delete m;
}

static fdp_status launch_apply(fdp_ctx *c, int width, int lanes, const uint32_t *moduli, const uint32_t *im,
                               const uint32_t *ib, uint32_t *om, uint32_t *ob, void *stream, ApplyArgs *a) {
  a->in_main = im;
  a->in_blk = ib;
  a->out_main = om;
  a->out_blk = ob;
  a->M = fdp::main_states(width);
  a->D = fdp::blocked_states(width);
  a->K = lanes;
  for (int i = 0; i < lanes; ++i) a->mod[i] = moduli[i];
  (void)c;
  (void)stream;
  return FDP_OK;
}

extern "C" fdp_status fdp_transfer_map_apply(fdp_ctx *c, const fdp_transfer_map *m, int lanes, const uint32_t *moduli,
                                             const uint32_t *d_in_main, const uint32_t *d_in_block,
                                             uint32_t *d_out_main, uint32_t *d_out_block, void *stream) {
  if (!c || !m) return FDP_ERR_ARGS;
  fdp_status s = check_apply(m->width, lanes, moduli, d_in_main, d_in_block, d_out_main, d_out_block);
  if (s != FDP_OK) return s;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fdp_cuda_status(e, "cudaSetDevice");
  ApplyArgs a{};
  launch_apply(c, m->width, lanes, moduli, d_in_main, d_in_block, d_out_main, d_out_block, stream, &a);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  csr_apply_kernel<<<grid_for(m->rows), 256, 0, st>>>(a, m->offsets, m->columns);
  return fdp_cuda_status(cudaGetLastError(), "csr apply");
}

extern "C" fdp_status fdp_reverse2_apply(fdp_ctx *c, int width, int p, int lanes, const uint32_t *moduli,
                                         const uint32_t *d_in_main, const uint32_t *d_in_block, uint32_t *d_out_main,
                                         uint32_t *d_out_block, void *stream) {
  if (!c || p < 2 || p >= width) {
    fdp_set_last_error("reverse2: need 2 <= p < width");
    return FDP_ERR_ARGS;
  }
  fdp_status s = check_apply(width, lanes, moduli, d_in_main, d_in_block, d_out_main, d_out_block);
  if (s != FDP_OK) return s;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fdp_cuda_status(e, "cudaSetDevice");
  const Counts *cnt = device_counts();
  if (!cnt) return FDP_ERR_HBM;
  ApplyArgs a{};
  launch_apply(c, width, lanes, moduli, d_in_main, d_in_block, d_out_main, d_out_block, stream, &a);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  reverse2_kernel<<<grid_for(a.M + a.D), 256, 0, st>>>(a, cnt, width, p);
  return fdp_cuda_status(cudaGetLastError(), "reverse2");
}

// ---- factorized transfer map over occupancy groups ------------------------
// The reference compiles one CSR per group shape and reuses it for every
// conjugate group (src/cuda/b300/factor_transfer_map.cuh:1-5, the proof in
// docs/results/frontier-compiled-2026-09-05.md): two groups whose fixed
// region carries the same number of R/L symbols differ only by where the N
// gaps sit, and moving the occupied symbols in order between those positions
// is a bijection that keeps the canonical order, the heights and every
// source of every cell that leaves the fixed region alone.  Here a group is
// the set of words whose bottom `fixed` positions are occupied (R or L)
// exactly at the set bits of a mask; cell p (and p-1 when paired) never
// touches those positions, and its closures only turn an R into an L or back,
// so each group is closed under the operator.  The CSR is built once, in the
// local ranks of the representative group (the bottom `occupied` positions
// set), and applied to up to max_groups groups at once: a gather moves each
// group's values into an arena with the groups interleaved as columns
// (row i of group g at i * G + g, the layout of factor_transfer_batch.cuh:13-47),
// the apply sums every row's sources column by column with one reduction per
// output, and a scatter writes the results back to their global ranks.

namespace {

Counts group_counts(int fixed, uint32_t occ) {
  Counts h;
  memset(&h, 0, sizeof(h));
  h.H[0][0] = 1;
  for (int w = 1; w <= FDP_MAXW; ++w) {
    const int q = w - 1;  // the position placed when w positions remain
    const bool n_ok = q >= fixed || !((occ >> q) & 1u), rl_ok = q >= fixed || ((occ >> q) & 1u);
    for (int k = 0; k < FDP_HT; ++k) {
      ull x = n_ok ? h.H[w - 1][k] : 0ull;
      if (rl_ok) {
        if (k > 0) x += h.H[w - 1][k - 1];
        if (k + 1 < FDP_HT) x += h.H[w - 1][k + 1];
      }
      h.H[w][k] = x;
    }
  }
  return h;
}

// The word of group `to` that corresponds to word w0 of group `from`: the
// occupied symbols of the fixed region keep their order and move to the set
// bits of `to`; positions from `fixed` up are unchanged.
__device__ __forceinline__ uint64_t move_occupied(uint64_t w0, uint32_t from, uint32_t to, int fixed) {
  uint64_t w = fixed ? (w0 & ~((1ull << (2 * fixed)) - 1ull)) : w0;
  while (from) {
    const int qa = __ffs(int(from)) - 1, qb = __ffs(int(to)) - 1;
    from &= from - 1u;
    to &= to - 1u;
    w |= uint64_t(get(w0, qa)) << (2 * qb);
  }
  return w;
}

struct GroupArgs {
  const Counts *gcounts, *full;
  int W, fixed;
  uint32_t occ0;
  ull gm, total;  // group main rows, main + blocked rows
  int G;
  const uint32_t *masks;
};

__global__ void group_gather_kernel(GroupArgs a, const uint32_t *in_main, const uint32_t *in_blk, uint32_t *arena,
                                    ull *ranks) {
  __shared__ ull sG[FDP_MAXW + 1][FDP_HT];
  __shared__ ull sF[FDP_MAXW + 1][FDP_HT];
  for (int k = threadIdx.x; k < (FDP_MAXW + 1) * FDP_HT; k += blockDim.x) {
    (&sG[0][0])[k] = (&a.gcounts->H[0][0])[k];
    (&sF[0][0])[k] = (&a.full->H[0][0])[k];
  }
  __syncthreads();
  const GroupSpace gs{sG, a.fixed, a.occ0};
  const ull n = a.total * ull(a.G);
  for (ull idx = ull(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += ull(gridDim.x) * blockDim.x) {
    const ull i = idx / ull(a.G);
    const int g = int(idx - i * ull(a.G));
    const bool is_main = i < a.gm;
    const int width = is_main ? a.W : a.W - 1;
    const uint64_t w = move_occupied(gs.unrank(is_main ? i : i - a.gm, width), a.occ0, a.masks[g], a.fixed);
    const ull r = rank_word_dev(w, width, sF);
    ranks[idx] = r;
    arena[idx] = is_main ? in_main[r] : in_blk[r];
  }
}

__global__ void group_apply_kernel(GroupArgs a, const uint32_t *arena_in, uint32_t *arena_out, const ull *offsets,
                                   const uint32_t *columns, uint32_t mod) {
  const ull n = a.total * ull(a.G);
  for (ull idx = ull(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += ull(gridDim.x) * blockDim.x) {
    const ull i = idx / ull(a.G);
    const ull g = idx - i * ull(a.G);
    ull sum = i < a.gm ? arena_in[idx] : 0ull;
    for (ull e = offsets[i]; e < offsets[i + 1]; ++e) sum += arena_in[ull(columns[e]) * ull(a.G) + g];
    arena_out[idx] = uint32_t(sum % mod);  // sum < 2^41: at most ~6W sources below 2^32
  }
}

__global__ void group_scatter_kernel(GroupArgs a, const uint32_t *arena_out, const ull *ranks, uint32_t *out_main,
                                     uint32_t *out_blk) {
  const ull n = a.total * ull(a.G);
  for (ull idx = ull(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += ull(gridDim.x) * blockDim.x) {
    const ull i = idx / ull(a.G);
    (i < a.gm ? out_main : out_blk)[ranks[idx]] = arena_out[idx];
  }
}

}  // namespace

struct fdp_factor_map {
  int device = 0, width = 0, p = 0, paired = 0, fixed = 0, occupied = 0, max_groups = 0;
  ull gm = 0, gd = 0, edges = 0;
  ull *offsets = nullptr;
  uint32_t *columns = nullptr;
  Counts *gcounts = nullptr;
  uint32_t *masks = nullptr, *arena_in = nullptr, *arena_out = nullptr;
  ull *ranks = nullptr;
  cudaEvent_t ev[4] = {};
  ~fdp_factor_map() {
    cudaSetDevice(device);
    for (void *q : {(void *)offsets, (void *)columns, (void *)gcounts, (void *)masks, (void *)arena_in,
                    (void *)arena_out, (void *)ranks})
      if (q) cudaFree(q);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  }
};

extern "C" fdp_status fdp_factor_map_build(fdp_ctx *c, int width, int p, int paired, int fixed, int occupied,
                                           int max_groups, fdp_factor_map **out) {
  if (!c || !out || width < 3 || width > FDP_MAXW || p < 1 || p >= width || (paired && p < 2) || fixed < 0 ||
      fixed > (paired ? p - 2 : p - 1) || fixed > 24 || occupied < 0 || occupied > fixed || max_groups < 1 ||
      max_groups > 32) {
    fdp_set_last_error(
        "factor_map_build: need 3 <= width <= 28, 1 <= p < width, 0 <= fixed <= p - 1 (p - 2 when paired, at most "
        "24), 0 <= occupied <= fixed, 1 <= max_groups <= 32");
    return FDP_ERR_ARGS;
  }
  *out = nullptr;
  const uint32_t occ0 = occupied ? (1u << occupied) - 1u : 0u;
  const Counts hg = group_counts(fixed, occ0);
  const ull gm = hg.H[width][1], gd = hg.H[width - 1][1], total = gm + gd;
  if (total == 0 || total > 0xffffffffull) {
    fdp_set_last_error(total ? "factor_map_build: group too large for 32-bit CSR columns"
                             : "factor_map_build: the group holds no word");
    return FDP_ERR_ARGS;
  }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fdp_cuda_status(e, "cudaSetDevice");
  const Counts *full = device_counts();
  if (!full) return FDP_ERR_HBM;
  auto map = std::make_unique<fdp_factor_map>();
  map->device = c->device;
  map->width = width;
  map->p = p;
  map->paired = paired ? 1 : 0;
  map->fixed = fixed;
  map->occupied = occupied;
  map->max_groups = max_groups;
  map->gm = gm;
  map->gd = gd;
  const size_t cells = size_t(total) * size_t(max_groups);
  if ((e = cudaMalloc(&map->gcounts, sizeof(Counts))) != cudaSuccess ||
      (e = cudaMemcpy(map->gcounts, &hg, sizeof(Counts), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMalloc(&map->masks, sizeof(uint32_t) * 32)) != cudaSuccess ||
      (e = cudaMalloc(&map->arena_in, sizeof(uint32_t) * cells)) != cudaSuccess ||
      (e = cudaMalloc(&map->arena_out, sizeof(uint32_t) * cells)) != cudaSuccess ||
      (e = cudaMalloc(&map->ranks, sizeof(ull) * cells)) != cudaSuccess)
    return fdp_cuda_status(e, "factor map buffers");
  for (cudaEvent_t &ev : map->ev)
    if ((e = cudaEventCreate(&ev)) != cudaSuccess) return fdp_cuda_status(e, "factor map events");
  const SpaceArgs sa{map->gcounts, fixed, occ0};
  fdp_status st = build_csr<true>(c, sa, gm, total, width, p, paired != 0, &map->offsets, &map->columns, &map->edges);
  if (st != FDP_OK) return st;
  *out = map.release();
  return FDP_OK;
}

extern "C" fdp_status fdp_factor_map_info(const fdp_factor_map *m, uint64_t *group_main, uint64_t *group_blocked,
                                          uint64_t *edges, uint64_t *device_bytes) {
  if (!m) return FDP_ERR_ARGS;
  const ull rows = m->gm + m->gd, cells = rows * ull(m->max_groups);
  if (group_main) *group_main = m->gm;
  if (group_blocked) *group_blocked = m->gd;
  if (edges) *edges = m->edges;
  if (device_bytes)
    *device_bytes = sizeof(ull) * (rows + 1) + sizeof(uint32_t) * m->edges + sizeof(Counts) + 4 * 32 +
                    cells * (2 * sizeof(uint32_t) + sizeof(ull));
  return FDP_OK;
}

extern "C" fdp_status fdp_factor_map_apply(fdp_ctx *c, const fdp_factor_map *m, uint32_t modulus, int groups,
                                           const uint32_t *masks, const uint32_t *d_in_main,
                                           const uint32_t *d_in_block, uint32_t *d_out_main, uint32_t *d_out_block,
                                           void *stream, double *phase_ms) {
  if (!c || !m || !masks || !d_in_main || !d_in_block || !d_out_main || !d_out_block || groups < 1 ||
      groups > m->max_groups) {
    fdp_set_last_error("factor_map_apply: need 1 <= groups <= max_groups, host masks and four device vectors");
    return FDP_ERR_ARGS;
  }
  if (modulus < 2) return FDP_ERR_MODULUS;
  for (int g = 0; g < groups; ++g)
    if (__builtin_popcount(masks[g]) != m->occupied || (m->fixed < 32 && (masks[g] >> m->fixed))) {
      fdp_set_last_error("factor_map_apply: every mask needs `occupied` set bits, all below `fixed`");
      return FDP_ERR_ARGS;
    }
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fdp_cuda_status(e, "cudaSetDevice");
  const Counts *full = device_counts();
  if (!full) return FDP_ERR_HBM;
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  if ((e = cudaMemcpyAsync(m->masks, masks, sizeof(uint32_t) * size_t(groups), cudaMemcpyHostToDevice, st)) !=
      cudaSuccess)
    return fdp_cuda_status(e, "factor map masks");
  GroupArgs a{m->gcounts, full, m->width, m->fixed, m->occupied ? (1u << m->occupied) - 1u : 0u,
              m->gm, m->gm + m->gd, groups, m->masks};
  const unsigned grid = grid_for(a.total * ull(groups));
  if (phase_ms) cudaEventRecord(m->ev[0], st);
  group_gather_kernel<<<grid, 256, 0, st>>>(a, d_in_main, d_in_block, m->arena_in, m->ranks);
  if (phase_ms) cudaEventRecord(m->ev[1], st);
  group_apply_kernel<<<grid, 256, 0, st>>>(a, m->arena_in, m->arena_out, m->offsets, m->columns, modulus);
  if (phase_ms) cudaEventRecord(m->ev[2], st);
  group_scatter_kernel<<<grid, 256, 0, st>>>(a, m->arena_out, m->ranks, d_out_main, d_out_block);
  if (phase_ms) cudaEventRecord(m->ev[3], st);
  if ((e = cudaGetLastError()) != cudaSuccess) return fdp_cuda_status(e, "factor map apply");
  if (phase_ms) {
    if ((e = cudaEventSynchronize(m->ev[3])) != cudaSuccess) return fdp_cuda_status(e, "factor map apply");
    for (int k = 0; k < 3; ++k) {
      float ms = 0;
      cudaEventElapsedTime(&ms, m->ev[k], m->ev[k + 1]);
      phase_ms[k] = ms;
    }
  }
  return FDP_OK;
}

extern "C" void fdp_factor_map_destroy(fdp_factor_map *m) { delete m; }
