// Dispatch of the templated kernels, per-width table upload, and the small
// operator-surface kernels (rank / unrank / ternary index).
#include <memory>

#include "fdp_host.h"
#include "fdp_launch.h"

namespace fdp {

int device_sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 148;
  return n;
}

cudaError_t upload_tables(int W, DevTables *out) {
  out->W = W;
  out->u64 = needs_u64(W);
  cudaError_t e;
  if (out->u64) {
    auto t = std::make_unique<WidthTables<uint64_t>>();
    build_width_tables<uint64_t>(W, t.get());
    if ((e = cudaMalloc(&out->ptr, sizeof(*t))) != cudaSuccess) return e;
    return cudaMemcpy(out->ptr, t.get(), sizeof(*t), cudaMemcpyHostToDevice);
  }
  auto t = std::make_unique<WidthTables<uint32_t>>();
  build_width_tables<uint32_t>(W, t.get());
  if ((e = cudaMalloc(&out->ptr, sizeof(*t))) != cudaSuccess) return e;
  return cudaMemcpy(out->ptr, t.get(), sizeof(*t), cudaMemcpyHostToDevice);
}

void free_tables(DevTables *t) {
  if (t->ptr) cudaFree(t->ptr);
  t->ptr = nullptr;
}

#define FDP_SWITCH_K(K, CALL)       \
  switch (K) {                      \
    case 1: return CALL(1);         \
    case 2: return CALL(2);         \
    case 3: return CALL(3);         \
    case 4: return CALL(4);         \
    case 5: return CALL(5);         \
    case 6: return CALL(6);         \
    case 7: return CALL(7);         \
    case 8: return CALL(8);         \
    case 9: return CALL(9);         \
    case 10: return CALL(10);       \
    case 11: return CALL(11);       \
    case 12: return CALL(12);       \
    case 13: return CALL(13);       \
    case 14: return CALL(14);       \
    case 15: return CALL(15);       \
    case 16: return CALL(16);       \
    default: return cudaErrorInvalidValue; \
  }

static cudaError_t launch_cell_k(const DevTables &t, int K, const CellArgs &a, const LaunchCfg &cfg, cudaStream_t s) {
  if (t.u64) {
#define CALL64(k) launch_cell_t<uint64_t, k>(a, cfg, s)
    FDP_SWITCH_K(K, CALL64)
#undef CALL64
  }
#define CALL32(k) launch_cell_t<uint32_t, k>(a, cfg, s)
  FDP_SWITCH_K(K, CALL32)
#undef CALL32
}

cudaError_t launch_cell(const DevTables &t, int K, const uint32_t *mods, uint32_t *main, uint32_t *blk, int p,
                        bool blk_in_zero, bool blk_out_p1, const LaunchCfg &cfg, cudaStream_t s) {
  if (!t.ptr || p < 1 || p >= t.W || K < 1 || K > kMaxLanes) return cudaErrorInvalidValue;
  CellArgs a{};
  a.tables = t.ptr;
  a.main = main;
  a.blk = blk;
  a.items = blocked_states(t.W);
  a.mstates = main_states(t.W);
  for (int i = 0; i < K; ++i) a.mod[i] = mods[i];
  a.W = t.W;
  a.p = p;
  a.blk_in_zero = blk_in_zero ? 1 : 0;
  a.blk_out_p1 = blk_out_p1 ? 1 : 0;
  const bool one_panel = (K == 1 || K == 2 || K == 4 || K == 8);
  if (one_panel || !cfg.split_panels) return launch_cell_k(t, K, a, cfg, s);
  // Every panel is an independent [N][PW] array: run each as its own K = PW problem.
  for (int l0 = 0; l0 < K;) {
    const int pw = (K - l0 >= 8) ? 8 : (K - l0 >= 4) ? 4 : (K - l0 >= 2) ? 2 : 1;
    CellArgs b = a;
    b.main = main + size_t(l0) * a.mstates;
    b.blk = blk + size_t(l0) * a.items;
    for (int i = 0; i < pw; ++i) b.mod[i] = mods[l0 + i];
    cudaError_t e = launch_cell_k(t, pw, b, cfg, s);
    if (e != cudaSuccess) return e;
    l0 += pw;
  }
  return cudaSuccess;
}

static cudaError_t first_row(const DevTables &t, int K, const uint32_t *mods, uint32_t *main,
                             unsigned long long *acc, bool dot, cudaStream_t s) {
  if (!t.ptr || K < 1 || K > kMaxLanes) return cudaErrorInvalidValue;
  FirstRowArgs a{};
  a.tables = t.ptr;
  a.main = main;
  a.acc = acc;
  a.mstates = main_states(t.W);
  for (int i = 0; i < K && mods; ++i) a.mod[i] = mods[i];
  a.W = t.W;
  if (t.u64) {
#define CALL64(k) launch_first_row_t<uint64_t, k>(a, dot, s)
    FDP_SWITCH_K(K, CALL64)
#undef CALL64
  }
#define CALL32(k) launch_first_row_t<uint32_t, k>(a, dot, s)
  FDP_SWITCH_K(K, CALL32)
#undef CALL32
}

cudaError_t launch_first_row_init(const DevTables &t, int K, uint32_t *main, cudaStream_t s) {
  return first_row(t, K, nullptr, main, nullptr, false, s);
}

__global__ void finalize_residues_kernel(const unsigned long long *acc, uint32_t *out, FirstRowArgs a, int k) {
  const int i = threadIdx.x;
  if (i < k) out[i] = uint32_t(acc[i] % a.mod[i]);
}

cudaError_t launch_first_row_dot(const DevTables &t, int K, const uint32_t *mods, const uint32_t *main,
                                 unsigned long long *acc, uint32_t *residues, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * K, s);
  if (e != cudaSuccess) return e;
  if ((e = first_row(t, K, mods, const_cast<uint32_t *>(main), acc, true, s)) != cudaSuccess) return e;
  FirstRowArgs a{};
  for (int i = 0; i < K; ++i) a.mod[i] = mods[i];
  finalize_residues_kernel<<<1, 32, 0, s>>>(acc, residues, a, K);
  return cudaGetLastError();
}

// ---- operator surface: canonical rank / unrank / ternary index ---------------
struct RankTable {
  unsigned long long H[FDP_MAXW + 1][FDP_HT];
};

__global__ void rank_words_kernel(const RankTable *T, int width, const uint64_t *words, uint64_t *ranks,
                                  uint64_t count) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += uint64_t(gridDim.x) * blockDim.x)
    ranks[i] = rank_dev<unsigned long long>(words[i], width, T->H);
}

__global__ void unrank_words_kernel(const RankTable *T, int width, const uint64_t *ranks, uint64_t *words,
                                    uint64_t count) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += uint64_t(gridDim.x) * blockDim.x) {
    unsigned long long r = ranks[i];
    uint64_t m = 0;
    int h = 1;
    for (int pos = width - 1; pos >= 0; --pos) {
      unsigned long long z = T->H[pos][h];
      if (r < z) continue;
      r -= z;
      if (h > 0) {
        z = T->H[pos][h - 1];
        if (r < z) {
          m |= uint64_t(SYM_R) << (2 * pos);
          --h;
          continue;
        }
        r -= z;
      }
      m |= uint64_t(SYM_L) << (2 * pos);
      ++h;
    }
    words[i] = m;
  }
}

// Ternary rank index (src/common/ternary_rank_index.hpp:6-15): read the two-bit
// digits N=0, R=1, L=2 of a legal segment as base-3 digits, least significant
// first.  A bijection from {N,R,L}^K onto [0, 3^K).
__global__ void ternary_index_kernel(const uint32_t *codes, uint32_t *index, uint64_t count) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t c = codes[i], x = 0, scale = 1;
    while (c) {
      x += (c & 3u) * scale;
      scale *= 3u;
      c >>= 2;
    }
    index[i] = x;
  }
}

static RankTable *rank_table() {
  static RankTable *d = nullptr;
  static int dev_of = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (d && dev_of == dev) return d;
  RankTable h;
  const CountTable &c = counts();
  for (int w = 0; w <= FDP_MAXW; ++w)
    for (int k = 0; k < FDP_HT; ++k) h.H[w][k] = c.H[w][k];
  RankTable *p = nullptr;
  if (cudaMalloc(&p, sizeof(h)) != cudaSuccess) return nullptr;
  if (cudaMemcpy(p, &h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
  d = p;
  dev_of = dev;
  return d;
}

static unsigned grid_for(uint64_t count) {
  uint64_t g = (count + 255) / 256, cap = uint64_t(device_sm_count()) * 8;
  return unsigned(g < 1 ? 1 : (g > cap ? cap : g));
}

cudaError_t launch_rank_words(int width, const uint64_t *words, uint64_t *ranks, uint64_t count, cudaStream_t s) {
  RankTable *T = rank_table();
  if (!T) return cudaErrorMemoryAllocation;
  if (!count) return cudaSuccess;
  rank_words_kernel<<<grid_for(count), 256, 0, s>>>(T, width, words, ranks, count);
  return cudaGetLastError();
}

cudaError_t launch_unrank_words(int width, const uint64_t *ranks, uint64_t *words, uint64_t count, cudaStream_t s) {
  RankTable *T = rank_table();
  if (!T) return cudaErrorMemoryAllocation;
  if (!count) return cudaSuccess;
  unrank_words_kernel<<<grid_for(count), 256, 0, s>>>(T, width, ranks, words, count);
  return cudaGetLastError();
}

cudaError_t launch_ternary_index(const uint32_t *codes, uint32_t *index, uint64_t count, cudaStream_t s) {
  if (!count) return cudaSuccess;
  ternary_index_kernel<<<grid_for(count), 256, 0, s>>>(codes, index, count);
  return cudaGetLastError();
}

}  // namespace fdp
