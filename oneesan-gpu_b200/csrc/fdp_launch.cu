// Dispatch of the templated kernels, per-width table upload, and the small
// operator-surface kernels (rank / unrank / ternary index).
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "fdp_host.h"
#include "fdp_launch.h"

namespace fdp {

int device_sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 148;
  return n;
}

cudaError_t upload_tables(int W, int cap, DevTables *out) {
  out->W = W;
  out->cap = cap;
  out->u64 = needs_u64(W);
  cudaError_t e;
  if (out->u64) {
    auto t = std::make_unique<WidthTables<uint64_t>>();
    build_width_tables<uint64_t>(W, t.get(), cap);
    if ((e = cudaMalloc(&out->ptr, sizeof(*t))) != cudaSuccess) return e;
    return cudaMemcpy(out->ptr, t.get(), sizeof(*t), cudaMemcpyHostToDevice);
  }
  auto t = std::make_unique<WidthTables<uint32_t>>();
  build_width_tables<uint32_t>(W, t.get(), cap);
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

// The scheduling fields of the launch for K lanes (after any split into
// spans or panels): warp chunk, and for small p grouping by centre type,
// with or without carry-over.
static CellArgs schedule_cell(const CellArgs &in, int K, const LaunchCfg &cfg) {
  CellArgs a = in;
  a.lane_items = cfg.lane_items < 1 ? 1 : cfg.lane_items;
  // A small problem runs at most as many items per lane as fill every
  // resident thread once: longer warp chunks would leave most SMs idle behind
  // a few warps' serial chains (n = 10, one lane: 2.65 -> 0.78 ms per pass).
  const uint64_t resident = uint64_t(device_sm_count()) * 4 * 256;  // 4 CTAs of 256 threads per SM
  const uint64_t fill = a.items / resident > 1 ? a.items / resident : 1;
  if (uint64_t(a.lane_items) > fill) a.lane_items = int(fill);
  int spans = 0;
  for (int l = 0; l < K; l = span_end_of(K, l)) ++spans;
  // Carry-over pays for one span; in a launch of several spans (closure
  // sources staged in shared memory) it was measured slower.
  const bool carry = cfg.compact_carry > 0 || (cfg.compact_carry == 0 && spans == 1);
  a.compact = a.p <= cfg.compact_max_p ? (carry ? 2 : 1) : 0;
  if (a.compact == 1) {
    int most = cfg.compact_items > 0 ? cfg.compact_items : (spans > 1 ? 2 : 4);
    if (most > FDP_REC_MAX_ITEMS) most = FDP_REC_MAX_ITEMS;
    if (a.lane_items > most) a.lane_items = most;
  } else if (a.compact == 2) {
    // The carry-over store does not grow with the chunk: compact_items sets
    // the chunk over which the prefix decode is shared.
    a.lane_items = cfg.compact_items > 0 ? cfg.compact_items : kCarryItems;
    if (uint64_t(a.lane_items) > fill) a.lane_items = int(fill);
  }
  return a;
}

static cudaError_t launch_cell_k(const DevTables &t, int K, const CellArgs &in, const LaunchCfg &cfg,
                                 cudaStream_t s) {
  const CellArgs a = schedule_cell(in, K, cfg);
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
                        bool blk_in_zero, bool blk_out_p1, const LaunchCfg &cfg, cudaStream_t s, uint64_t *kernels) {
  if (!t.ptr || p < 1 || p >= t.W || K < 1 || K > kMaxLanes) return cudaErrorInvalidValue;
  CellArgs a{};
  a.tables = t.ptr;
  a.main = main;
  a.blk = blk;
  a.items = blocked_states_capped(t.W, t.cap);
  a.mstates = main_states_capped(t.W, t.cap);
  for (int i = 0; i < K; ++i) a.mod[i] = mods[i];
  a.W = t.W;
  a.p = p;
  a.cap = t.cap;
  a.blk_in_zero = blk_in_zero ? 1 : 0;
  a.blk_out_p1 = blk_out_p1 ? 1 : 0;
  a.share_prefix = (t.W - 1 - p) >= cfg.share_min ? 1 : 0;
  const bool one_panel = (K == 1 || K == 2 || K == 4 || K == 8);
  if (K > 8 && p >= cfg.split_spans_min_p && !cfg.split_panels) {
    // Each span (panels of at most 8 lanes together) is laid out exactly as a
    // lane count of its own width at its first panel's offset, so it runs as
    // an independent single-span problem: one launch per span, each decoding
    // the items again but streaming one span without staged closure sources.
    for (int l0 = 0; l0 < K;) {
      const int le = span_end_of(K, l0);
      CellArgs b = a;
      b.main = main + size_t(l0) * a.mstates;
      b.blk = blk + size_t(l0) * a.items;
      for (int i = 0; i < le - l0; ++i) b.mod[i] = mods[l0 + i];
      cudaError_t e = launch_cell_k(t, le - l0, b, cfg, s);
      if (e != cudaSuccess) return e;
      if (kernels) ++*kernels;
      l0 = le;
    }
    return cudaSuccess;
  }
  if (one_panel || !cfg.split_panels) {
    if (kernels) ++*kernels;
    return launch_cell_k(t, K, a, cfg, s);
  }
  // Every panel is an independent [N][PW] array: run each as its own K = PW problem.
  for (int l0 = 0; l0 < K;) {
    const int pw = (K - l0 >= 8) ? 8 : (K - l0 >= 4) ? 4 : (K - l0 >= 2) ? 2 : 1;
    CellArgs b = a;
    b.main = main + size_t(l0) * a.mstates;
    b.blk = blk + size_t(l0) * a.items;
    for (int i = 0; i < pw; ++i) b.mod[i] = mods[l0 + i];
    cudaError_t e = launch_cell_k(t, pw, b, cfg, s);
    if (e != cudaSuccess) return e;
    if (kernels) ++*kernels;
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

// ---- height-bounded prefix: row-0 fill and in-place expansion ------------------
__global__ void fill_ones_kernel(uint32_t *a, uint64_t words) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < words; i += uint64_t(gridDim.x) * blockDim.x)
    a[i] = 1u;
}

cudaError_t launch_fill_ones(uint32_t *a, uint64_t words, cudaStream_t s) {
  if (!words) return cudaSuccess;
  uint64_t g = (words + 255) / 256, cap = uint64_t(device_sm_count()) * 8;
  fill_ones_kernel<<<unsigned(g < cap ? g : cap), 256, 0, s>>>(a, words);
  return cudaGetLastError();
}

struct CapTable {
  unsigned long long H[FDP_MAXW + 1][FDP_HT];
};

// dst[rank_to(w_i) * PW + l] = tmp[(i - lo) * PW + l] for the words w_i of the
// `from` space with index i in [lo, hi).  Each warp takes chunks of 32 x 8
// consecutive indices; the top symbols the chunk's first and last words share
// are decoded once (ranks are lexicographic from the top), each lane walks the
// rest, and panels move as whole vectors.
template <int PW>
__global__ void __launch_bounds__(256) expand_scatter_kernel(const CapTable *from, const CapTable *to, int W,
                                                             uint64_t lo, uint64_t hi, const uint32_t *tmp,
                                                             uint32_t *dst) {
  __shared__ unsigned long long sf[FDP_MAXW + 1][FDP_HT], st[FDP_MAXW + 1][FDP_HT];
  for (int i = threadIdx.x; i < (FDP_MAXW + 1) * FDP_HT; i += blockDim.x) {
    (&sf[0][0])[i] = (&from->H[0][0])[i];
    (&st[0][0])[i] = (&to->H[0][0])[i];
  }
  __syncthreads();
  constexpr uint64_t kChunk = 32 * 8;
  const uint64_t n = hi - lo, wpb = blockDim.x >> 5, lane = threadIdx.x & 31;
  const uint64_t step = uint64_t(gridDim.x) * wpb * kChunk;
  for (uint64_t cb = (uint64_t(blockIdx.x) * wpb + (threadIdx.x >> 5)) * kChunk; cb < n; cb += step) {
    const uint64_t ce = n - cb > kChunk ? cb + kChunk : n;  // chunk [cb, ce) of [0, n)
    uint64_t r0 = lo + cb, r1 = lo + ce - 1, j0 = 0;
    int h = 1, pos = W - 1;
    for (; pos >= 0; --pos) {  // the shared top symbols (warp-uniform)
      uint64_t a0 = r0, a1 = r1, jj = j0, b1 = 0;
      int h0 = h, h1 = h;
      expand_step(sf, st, pos, a0, jj, h0);
      expand_step(sf, st, pos, a1, b1, h1);
      if (h0 != h1) break;  // the symbols differ (N keeps h, R lowers it, L raises it)
      r0 = a0;
      r1 = a1;
      j0 = jj;
      h = h0;
    }
    const uint64_t sub = lo + cb - r0;  // rank consumed by the shared symbols
    for (uint64_t i = cb + lane; i < ce; i += 32) {
      uint64_t r = lo + i - sub, j = j0;
      int hh = h;
      for (int q = pos; q >= 0; --q) expand_step(sf, st, q, r, j, hh);
      const uint32_t *s = tmp + size_t(i) * PW;
      uint32_t *d = dst + size_t(j) * PW;
      if constexpr (PW == 8) {
        reinterpret_cast<uint4 *>(d)[0] = reinterpret_cast<const uint4 *>(s)[0];
        reinterpret_cast<uint4 *>(d)[1] = reinterpret_cast<const uint4 *>(s)[1];
      } else if constexpr (PW == 4) {
        *reinterpret_cast<uint4 *>(d) = *reinterpret_cast<const uint4 *>(s);
      } else if constexpr (PW == 2) {
        *reinterpret_cast<uint2 *>(d) = *reinterpret_cast<const uint2 *>(s);
      } else {
        *d = *s;
      }
    }
    if (n - cb <= step) break;
  }
}

static const CapTable *cap_table(int cap) {
  static std::map<std::pair<int, int>, CapTable *> tabs;  // (device, cap) -> table
  static std::mutex mu;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto key = std::make_pair(dev, cap);
  auto it = tabs.find(key);
  if (it != tabs.end()) return it->second;
  CapTable h;
  const CountTable &c = counts_capped(cap);
  for (int w = 0; w <= FDP_MAXW; ++w)
    for (int k = 0; k < FDP_HT; ++k) h.H[w][k] = c.H[w][k];
  CapTable *p = nullptr;
  if (cudaMalloc(&p, sizeof(h)) != cudaSuccess) return nullptr;
  if (cudaMemcpy(p, &h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
  tabs[key] = p;
  return p;
}

cudaError_t prepare_expand_tables(const std::vector<int> &caps) {
  for (int cap : caps)
    if (!cap_table(cap)) return cudaErrorMemoryAllocation;
  return cudaSuccess;
}

cudaError_t enqueue_expand(const DevTables &from, const DevTables &to, int K, uint32_t *a, uint32_t *tmp,
                           uint64_t tmp_words, cudaStream_t s, uint64_t *launches) {
  const int W = from.W;
  const uint64_t Nf = main_states_capped(W, from.cap), Nt = main_states_capped(W, to.cap);
  const CapTable *tf = cap_table(from.cap), *tt = cap_table(to.cap);
  if (!tf || !tt) return cudaErrorMemoryAllocation;
  // Panels (first lane, width) of the K-lane layout, last panel first.
  std::vector<std::pair<int, int>> panels;
  for (int l0 = 0; l0 < K;) {
    const int pw = (K - l0 >= 8) ? 8 : (K - l0 >= 4) ? 4 : (K - l0 >= 2) ? 2 : 1;
    panels.push_back({l0, pw});
    l0 += pw;
  }
  for (size_t pi = panels.size(); pi-- > 0;) {
    const int l0 = panels[pi].first, pw = panels[pi].second;
    uint32_t *src = a + size_t(l0) * Nf, *dst = a + size_t(l0) * Nt;
    const uint64_t chunk = tmp_words / uint64_t(pw);
    if (!chunk) return cudaErrorInvalidValue;
    uint64_t hi = Nf, top = Nt;  // `top`: new index of the chunk above (already placed)
    while (hi > 0) {
      const uint64_t lo = hi > chunk ? hi - chunk : 0;
      const uint64_t nlo = rank_word(unrank_word(lo, W, from.cap), W, to.cap);
      cudaError_t e = cudaMemcpyAsync(tmp, src + size_t(lo) * pw, size_t(hi - lo) * pw * 4, cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return e;
      if ((e = cudaMemsetAsync(dst + size_t(nlo) * pw, 0, size_t(top - nlo) * pw * 4, s)) != cudaSuccess) return e;
      const uint64_t n = hi - lo;
      uint64_t g = (n + 255) / 256, gc = uint64_t(device_sm_count()) * 8;
      const unsigned grid = unsigned(g < gc ? g : gc);
      if (pw == 8) expand_scatter_kernel<8><<<grid, 256, 0, s>>>(tf, tt, W, lo, hi, tmp, dst);
      else if (pw == 4) expand_scatter_kernel<4><<<grid, 256, 0, s>>>(tf, tt, W, lo, hi, tmp, dst);
      else if (pw == 2) expand_scatter_kernel<2><<<grid, 256, 0, s>>>(tf, tt, W, lo, hi, tmp, dst);
      else expand_scatter_kernel<1><<<grid, 256, 0, s>>>(tf, tt, W, lo, hi, tmp, dst);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      if (launches) ++*launches;
      top = nlo;
      hi = lo;
    }
  }
  return cudaSuccess;
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

// The count table of the rank / unrank kernels, uploaded once per device.
static RankTable *rank_table() {
  static std::mutex mu;
  static std::map<int, RankTable *> per_dev;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  auto it = per_dev.find(dev);
  if (it != per_dev.end()) return it->second;
  RankTable h;
  const CountTable &c = counts();
  for (int w = 0; w <= FDP_MAXW; ++w)
    for (int k = 0; k < FDP_HT; ++k) h.H[w][k] = c.H[w][k];
  RankTable *p = nullptr;
  if (cudaMalloc(&p, sizeof(h)) != cudaSuccess) return nullptr;
  if (cudaMemcpy(p, &h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(p);
    return nullptr;
  }
  per_dev[dev] = p;
  return p;
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

// Chunked conversion (the reference's GRIDFP_TRIT_CHUNK, R2.cu:23-55): a table
// of the ternary index of every code of `CH` symbols (4^CH entries, built in
// shared memory by each block), so a code of up to 16 symbols converts with
// one table read per chunk: index = sum_k T[chunk_k] x (3^CH)^k.
template <int CH>
__global__ void ternary_index_chunked_kernel(const uint32_t *codes, uint32_t *index, uint64_t count) {
  constexpr uint32_t n = 1u << (2 * CH), mask = n - 1u;
  constexpr uint32_t radix = CH == 7 ? 2187u : 81u;
  __shared__ uint16_t T[n];
  for (uint32_t c = threadIdx.x; c < n; c += blockDim.x) {
    uint32_t x = 0, scale = 1, v = c;
    for (int k = 0; k < CH; ++k) {
      x += (v & 3u) * scale;
      scale *= 3u;
      v >>= 2;
    }
    T[c] = uint16_t(x);
  }
  __syncthreads();
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t c = codes[i], x = 0, scale = 1;
    for (int off = 0; off < 16 && c; off += CH) {
      x += uint32_t(T[c & mask]) * scale;
      scale *= radix;
      c >>= 2 * CH;
    }
    index[i] = x;
  }
}

cudaError_t launch_ternary_index_chunked(int chunk, const uint32_t *codes, uint32_t *index, uint64_t count,
                                         cudaStream_t s) {
  if (chunk != 4 && chunk != 7) return cudaErrorInvalidValue;
  if (!count) return cudaSuccess;
  if (chunk == 4) ternary_index_chunked_kernel<4><<<grid_for(count), 256, 0, s>>>(codes, index, count);
  else ternary_index_chunked_kernel<7><<<grid_for(count), 256, 0, s>>>(codes, index, count);
  return cudaGetLastError();
}

cudaError_t launch_ternary_index(const uint32_t *codes, uint32_t *index, uint64_t count, cudaStream_t s) {
  if (!count) return cudaSuccess;
  ternary_index_kernel<<<grid_for(count), 256, 0, s>>>(codes, index, count);
  return cudaGetLastError();
}

}  // namespace fdp
