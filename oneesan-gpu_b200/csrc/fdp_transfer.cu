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

// Sources (indices into [0, M+D)) of row i at cell p; main rows emit i first.
template <class Emit>
__device__ void step_sources(ull i, ull M, int W, int p, const ull (*Hm)[FDP_HT], Emit &&emit) {
  if (i < M) {
    const uint64_t t = unrank_word_dev(i, W, Hm);
    emit(i);
    auto main_src = [&](uint64_t s) { emit(rank_word_dev(s, W, Hm)); };
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
    if (a == SYM_N) emit(M + rank_word_dev(drop_at(t, p), W - 1, Hm));
    return;
  }
  if (p < 2) return;  // no blocked output at p = 1
  const uint64_t bw = unrank_word_dev(i - M, W - 1, Hm);
  const uint64_t u = insert_at(bw, p, fdp::SYM_N);
  const uint32_t c = get(bw, p - 1);
  auto main_src = [&](uint64_t s) { emit(rank_word_dev(s, W, Hm)); };
  if (c != fdp::SYM_N) {
    main_src(u);
    return;
  }
  if (height_above(u, W, p) >= 1) main_src(put_pair(u, p, fdp::SYM_R, fdp::SYM_L));
  ll_closures(u, p, main_src);
  rr_closures(u, W, p, main_src);
}

template <class Emit>
__device__ void sources(ull i, ull M, int W, int p, bool paired, const ull (*Hm)[FDP_HT], Emit &&emit) {
  if (!paired) {
    step_sources(i, M, W, p, Hm, emit);
    return;
  }
  step_sources(i, M, W, p - 1, Hm, [&](ull j) { step_sources(j, M, W, p, Hm, emit); });
}

__device__ void load_counts(ull (*sH)[FDP_HT], const Counts *c) {
  for (int k = threadIdx.x; k < (FDP_MAXW + 1) * FDP_HT; k += blockDim.x) (&sH[0][0])[k] = (&c->H[0][0])[k];
  __syncthreads();
}

__global__ void csr_count_kernel(const Counts *c, ull M, ull total, int W, int p, bool paired, ull *rowlen) {
  __shared__ ull sH[FDP_MAXW + 1][FDP_HT];
  load_counts(sH, c);
  for (ull i = ull(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += ull(gridDim.x) * blockDim.x) {
    ull n = 0;
    sources(i, M, W, p, paired, sH, [&](ull) { ++n; });
    rowlen[i] = n - (i < M ? 1 : 0);
  }
}

__global__ void csr_fill_kernel(const Counts *c, ull M, ull total, int W, int p, bool paired, const ull *offsets,
                                uint32_t *columns, ull *errors) {
  __shared__ ull sH[FDP_MAXW + 1][FDP_HT];
  load_counts(sH, c);
  ull bad = 0;
  for (ull i = ull(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += ull(gridDim.x) * blockDim.x) {
    ull pos = offsets[i];
    const ull end = offsets[i + 1];
    bool first = i < M;
    sources(i, M, W, p, paired, sH, [&](ull j) {
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
  const ull total = a.M + a.D;
  for (ull i = ull(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += ull(gridDim.x) * blockDim.x) {
    ull sum[16];
    for (int l = 0; l < a.K; ++l) sum[l] = 0;
    sources(i, a.M, W, p, true, sH, [&](ull j) {
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
  ull *err = nullptr;
  if ((e = cudaMalloc(&map->offsets, sizeof(ull) * (total + 1))) != cudaSuccess) return fdp_cuda_status(e, "csr offsets");
  if ((e = cudaMalloc(&err, sizeof(ull))) != cudaSuccess) {
    cudaFree(map->offsets);
    return fdp_cuda_status(e, "csr errors");
  }
  auto fail = [&](cudaError_t ce, const char *what) {
    cudaFree(err);
    if (map->offsets) cudaFree(map->offsets);
    if (map->columns) cudaFree(map->columns);
    return fdp_cuda_status(ce, what);
  };
  csr_count_kernel<<<grid_for(total), 256, 0, c->stream>>>(cnt, M, total, width, p, paired != 0, map->offsets);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "csr count");
  std::vector<ull> off(total + 1);
  if ((e = cudaMemcpyAsync(off.data(), map->offsets, sizeof(ull) * total, cudaMemcpyDeviceToHost, c->stream)) !=
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
  map->edges = run;
  if ((e = cudaMemcpyAsync(map->offsets, off.data(), sizeof(ull) * (total + 1), cudaMemcpyHostToDevice, c->stream)) !=
      cudaSuccess)
    return fail(e, "csr offsets copy");
  if ((e = cudaMalloc(&map->columns, sizeof(uint32_t) * (run ? run : 1))) != cudaSuccess) return fail(e, "csr columns");
  cudaMemsetAsync(err, 0, sizeof(ull), c->stream);
  csr_fill_kernel<<<grid_for(total), 256, 0, c->stream>>>(cnt, M, total, width, p, paired != 0, map->offsets,
                                                          map->columns, err);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "csr fill");
  ull bad = 0;
  if ((e = cudaMemcpyAsync(&bad, err, sizeof(ull), cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess)
    return fail(e, "csr verify copy");
  if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return fail(e, "csr fill sync");
  cudaFree(err);
  if (bad) {
    cudaFree(map->offsets);
    cudaFree(map->columns);
    fdp_set_last_error("transfer_map_build: the fill pass disagreed with the count pass");
    return FDP_ERR_CUDA;
  }
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
