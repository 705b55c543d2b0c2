// Row-k initialiser, device half: the fill of fdp_rowinit.h on the GPU.
//
//   prefix levels : one warp per prefix, v_child[q'] = sum over the automaton
//                   edges into q' of v_parent[q] x weight (mod p per lane);
//   suffix levels : one warp per completion, u[q] = sum over the edges out of
//                   q of weight x u_child[q'];
//   products      : per end height h, out[base_x + j] = v_x . U_h[j], on the
//                   tensor cores (rowinit_mma_kernel: u8 limbs, s32
//                   accumulators in tensor memory, K <= 1024) or on the CUDA
//                   cores (rowinit_product_kernel: 64 prefixes x 64
//                   completions per tile, suffix values split into 16-bit
//                   halves so that every partial sum stays below 2^64 for up
//                   to 2^16 terms); one Barrett reduction per output either way.
// Scratch (two prefix levels, two suffix levels) is the caller's; the state
// vector is written in the lane-panel layout of the cell kernels.
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "fdp_launch.h"
#include "fdp_rowinit.h"
#include "fdp_rowinit_dev.h"

namespace fdp {

namespace {

constexpr int kH = 8;  // heights 0..7

struct Lanes {
  uint32_t p[16];
  unsigned long long m[16];  // floor((2^64 - 1) / p)
  uint64_t off[16];          // word offset of lane l's panel: L0 * N + (l - L0)
  int pw[16];                // panel width of lane l
  uint32_t c8[16][7];        // 2^(8s) mod p, s = 0..6 (tensor-core product's limb shifts)
  // Lane groups of the tensor-core product: up to four lanes of one panel,
  // adjacent in every state's panel words.
  int ngroups;
  int grp_lane0[16], grp_n[16];
};

__device__ __forceinline__ uint32_t red64(unsigned long long x, uint32_t p, unsigned long long m) {
  unsigned long long q = __umul64hi(x, m);
  unsigned long long r = x - q * p;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    if (r >= p) r -= p;
  return uint32_t(r);
}

struct AutDev {
  const int *gid;         // [hoff[h] + q] -> global state id
  const int *first_off;   // [3 + 1]
  const int *first_to;    // local index
  const uint32_t *first_w;
  const int *fwd_off;     // [3 * (n + 1)] by (sym, target global id): edges into it
  const int *fwd_from;    // local index of the source
  const uint32_t *fwd_w;
  const int *bwd_off;     // [3 * (n + 1)] by (sym, source global id): edges out of it
  const int *bwd_to;      // local index of the target
  const uint32_t *bwd_w;
  const uint32_t *last_w; // [3 * n] by (sym, source global id)
  int n;
  int K[kH], hoff[kH];
};

struct LevelArgs {
  uint64_t base[kH];  // word offset of height h's block (all lanes)
  uint64_t cnt[kH];   // rows (prefix levels) or columns (suffix levels) of height h
};

__global__ void __launch_bounds__(256) rowinit_prefix_kernel(AutDev a, Lanes ln, int L, int first, int nprefix,
                                                             const int32_t *parent, const uint8_t *sym,
                                                             const uint8_t *height, const int32_t *row,
                                                             const uint8_t *pheight, const int32_t *prow,
                                                             LevelArgs cur, LevelArgs prev, const uint32_t *vin,
                                                             uint32_t *vout) {
  const int lane = threadIdx.x & 31;
  const int warps = int((gridDim.x * blockDim.x) >> 5);
  for (int i = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < nprefix; i += warps) {
    const int h = height[i], s = sym[i], K = a.K[h];
    const uint64_t ob = cur.base[h] + uint64_t(row[i]) * uint64_t(K);
    const uint64_t lstride = cur.cnt[h] * uint64_t(K);
    int hp = 0;
    uint64_t ib = 0, istride = 0;
    if (!first) {
      const int pi = parent[i];
      hp = pheight[pi];
      ib = prev.base[hp] + uint64_t(prow[pi]) * uint64_t(a.K[hp]);
      istride = prev.cnt[hp] * uint64_t(a.K[hp]);
    }
    for (int q = lane; q < K; q += 32) {
      unsigned long long acc[16];
      for (int l = 0; l < L; ++l) acc[l] = 0;
      if (first) {
        for (int e = a.first_off[s]; e < a.first_off[s + 1]; ++e)
          if (a.first_to[e] == q)
            for (int l = 0; l < L; ++l) acc[l] += a.first_w[e];
      } else {
        const int t = a.gid[a.hoff[h] + q];
        const int *off = a.fwd_off + s * (a.n + 1);
        for (int e = off[t]; e < off[t + 1]; ++e) {
          const int src = a.fwd_from[e];
          const uint32_t w = a.fwd_w[e];
          for (int l = 0; l < L; ++l) acc[l] += (unsigned long long)vin[ib + uint64_t(l) * istride + src] * w;
        }
      }
      for (int l = 0; l < L; ++l) vout[ob + uint64_t(l) * lstride + q] = red64(acc[l], ln.p[l], ln.m[l]);
    }
  }
}

// C[k][g] for the two suffix levels a kernel touches.
struct SufCounts {
  uint64_t cur[kH], prev[kH];
};

__global__ void __launch_bounds__(256) rowinit_suffix_kernel(AutDev a, Lanes ln, int L, int first_level, int hmax,
                                                             SufCounts c, LevelArgs cur, LevelArgs prev,
                                                             const uint32_t *uin, uint32_t *uout) {
  const int lane = threadIdx.x & 31;
  uint64_t total = 0;
  for (int g = 0; g <= hmax; ++g) total += c.cur[g];
  const uint64_t warps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t col = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; col < total; col += warps) {
    int g = 0;
    uint64_t j = col;
    while (j >= c.cur[g]) j -= c.cur[g++];
    const int K = a.K[g];
    if (!K) continue;
    const uint64_t ob = cur.base[g] + j * uint64_t(K);
    const uint64_t lstride = cur.cnt[g] * uint64_t(K);
    int s, gc = g;
    uint64_t jc = j;
    if (first_level) {
      s = g == 0 ? 0 : 1;  // one position left: N from 0 or R from 1
    } else if (jc < c.prev[g]) {
      s = 0;
    } else {
      jc -= c.prev[g];
      const uint64_t cr = g >= 1 ? c.prev[g - 1] : 0;
      if (jc < cr) {
        s = 1;
        gc = g - 1;
      } else {
        jc -= cr;
        s = 2;
        gc = g + 1;
      }
    }
    for (int q = lane; q < K; q += 32) {
      const int src = a.gid[a.hoff[g] + q];
      unsigned long long acc[16];
      for (int l = 0; l < L; ++l) acc[l] = 0;
      if (first_level) {
        const uint32_t w = a.last_w[s * a.n + src];
        for (int l = 0; l < L; ++l) acc[l] = w;
      } else if (gc <= hmax) {
        const uint64_t ib = prev.base[gc] + jc * uint64_t(a.K[gc]);
        const uint64_t istride = prev.cnt[gc] * uint64_t(a.K[gc]);
        const int *off = a.bwd_off + s * (a.n + 1);
        for (int e = off[src]; e < off[src + 1]; ++e) {
          const int dst = a.bwd_to[e];
          const uint32_t w = a.bwd_w[e];
          for (int l = 0; l < L; ++l) acc[l] += (unsigned long long)uin[ib + uint64_t(l) * istride + dst] * w;
        }
      }
      for (int l = 0; l < L; ++l) uout[ob + uint64_t(l) * lstride + q] = red64(acc[l], ln.p[l], ln.m[l]);
    }
  }
}

// out[base[i] + j] = V[i] . U[j] for one end height: V is n rows x K, U is C
// columns x K (both K-contiguous, per lane at stride n*K / C*K).
constexpr int TM = 64, TN = 64, TQ = 16;
__global__ void __launch_bounds__(256) rowinit_product_kernel(Lanes ln, int L, int K, uint64_t n, uint64_t C,
                                                              const uint32_t *V, const uint32_t *U,
                                                              const uint64_t *base, uint32_t *out) {
  __shared__ __align__(16) uint32_t As[TQ][TM], Bl[TQ][TN], Bh[TQ][TN];
  const uint64_t tiles_n = (C + TN - 1) / TN;
  const uint64_t tile = blockIdx.x;
  const uint64_t i0 = (tile / tiles_n) * TM, j0 = (tile % tiles_n) * TN;
  const int t = threadIdx.x, ty = t >> 4, tx = t & 15;
  for (int l = 0; l < L; ++l) {
    const uint32_t *Vl = V + uint64_t(l) * n * uint64_t(K);
    const uint32_t *Ul = U + uint64_t(l) * C * uint64_t(K);
    unsigned long long lo[4][4], hi[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) lo[r][c] = hi[r][c] = 0;
    for (int q0 = 0; q0 < K; q0 += TQ) {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int e = t + 256 * r, rr = e / TQ, qq = e % TQ;
        const uint64_t gi = i0 + uint64_t(rr), gj = j0 + uint64_t(rr);
        const int gq = q0 + qq;
        As[qq][rr] = (gi < n && gq < K) ? Vl[gi * uint64_t(K) + uint64_t(gq)] : 0u;
        const uint32_t b = (gj < C && gq < K) ? Ul[gj * uint64_t(K) + uint64_t(gq)] : 0u;
        Bl[qq][rr] = b & 0xffffu;
        Bh[qq][rr] = b >> 16;
      }
      __syncthreads();
#pragma unroll
      for (int qq = 0; qq < TQ; ++qq) {
        const uint4 av = *reinterpret_cast<const uint4 *>(&As[qq][ty * 4]);
        const uint4 bl = *reinterpret_cast<const uint4 *>(&Bl[qq][tx * 4]);
        const uint4 bh = *reinterpret_cast<const uint4 *>(&Bh[qq][tx * 4]);
        const uint32_t ar[4] = {av.x, av.y, av.z, av.w}, blr[4] = {bl.x, bl.y, bl.z, bl.w},
                       bhr[4] = {bh.x, bh.y, bh.z, bh.w};
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            lo[r][c] += (unsigned long long)ar[r] * blr[c];
            hi[r][c] += (unsigned long long)ar[r] * bhr[c];
          }
      }
      __syncthreads();
    }
    const uint32_t p = ln.p[l];
    const unsigned long long m = ln.m[l];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const uint64_t gi = i0 + uint64_t(ty * 4 + r);
      if (gi >= n) continue;
      const uint64_t b0 = base[gi];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const uint64_t gj = j0 + uint64_t(tx * 4 + c);
        if (gj >= C) continue;
        const unsigned long long h16 = (unsigned long long)red64(hi[r][c], p, m) << 16;
        const uint32_t v = red64(red64(lo[r][c], p, m) + h16, p, m);
        out[ln.off[l] + (b0 + gj) * uint64_t(ln.pw[l])] = v;
      }
    }
  }
}

// The same products on the 5th-generation tensor cores (tcgen05, kind::i8).
// Every value is split into four u8 limbs, v = sum_i 2^(8i) v_i; the 16 limb
// products accumulate by shift s = i + j into seven s32 accumulators in tensor
// memory (7 x 64 of the 512 columns), so out = sum_s 2^(8s) G_s mod p.  A
// group sums at most 4 x K x 255^2 < 2^28 for K <= 1024 (larger K uses the
// CUDA-core product), so sum_s G_s (2^(8s) mod p) fits 64 bits and each output
// needs one reduction.
//
// Operands are first packed (rowinit_pack_kernel) into the tensor cores'
// shared-memory layout, one contiguous tile per 32-wide K step: K-major, no
// swizzle, core matrices of 8 rows x 16 bytes, 256 bytes between 8-row
// groups, 128 bytes between the two 16-byte K halves, the four limbs one after
// the other (128-row A tiles of 16 KB, 64-row B tiles of 8 KB).  The product
// kernel streams them with bulk copies into a 4-stage ring: thread 0 issues
// the copies (each stage completes an mbarrier by bytes), the MMAs of a stage
// as soon as it has landed, and commits them to the stage's "empty" mbarrier,
// so the copies of the next stages overlap the MMAs.
//
// A work item is one 128 x 64 tile for a group of up to four lanes of one
// panel (the lanes whose words of a state are adjacent in memory).  The lanes
// of the group are multiplied one after another; after each, warps 4..7 read
// the seven accumulator groups of their rows out of tensor memory, hand it
// back (an mbarrier the issuer waits on before the next lane's MMAs), reduce
// mod p and park the residues in shared memory as [row][column][lane].  Once
// the group is complete each warp writes its 32 rows: per row 64 consecutive
// states, every state's group of lanes one 16-, 8- or 4-byte store, so a warp
// store covers one contiguous run of the panel instead of 32 scattered words.
// Items run in bands of eight row tiles so that a band's column tiles are
// read from memory once for all eight.  Every wait is bounded.  One CTA per SM
// (it holds all 512 tensor-memory columns and 226 KB of shared memory).
constexpr int MM = 128, MN = 64, MK = 32;
constexpr int A_LIMB = MM * MK, B_LIMB = MN * MK;         // bytes of one limb's tile per K step
constexpr int A_TILE = 4 * A_LIMB, B_TILE = 4 * B_LIMB;   // 16 KB, 8 KB
constexpr int NST = 4;                                    // ring stages
constexpr uint32_t kIdescI8 = (2u << 4) | (uint32_t(MN >> 3) << 17) | (uint32_t(MM >> 4) << 24);  // S32 += U8 x U8, K-major
constexpr uint32_t kIdescN256 = (2u << 4) | (uint32_t(4 * MN >> 3) << 17) | (uint32_t(MM >> 4) << 24);
constexpr uint32_t kIdescN192 = (2u << 4) | (uint32_t(3 * MN >> 3) << 17) | (uint32_t(MM >> 4) << 24);
constexpr uint32_t kTmemCols = 512;
constexpr int SROW = MN * 4 + 4;                          // staged words per row: 64 states x 4 lanes, padded
constexpr size_t kRingBytes = size_t(NST) * (A_TILE + B_TILE);
constexpr size_t kMmaSmem = kRingBytes + size_t(MM) * SROW * 4;  // 96 KB ring + 130 KB staging
constexpr int RBAND = 8;                                  // row tiles per band of the item order

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  return uint64_t((saddr >> 4) & 0x3fffu) | (uint64_t(128 >> 4) << 16) | (uint64_t(256 >> 4) << 32) |
         (uint64_t(1) << 46);
}

// D[tmem] (+)= A x B^T, M = 128, u8 x u8 -> s32; `acc` = 0 overwrites D.
__device__ __forceinline__ void mma_i8(uint32_t d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred PRED_enable_input_d;\n\t"
      "setp.ne.b32 PRED_enable_input_d, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, PRED_enable_input_d;\n\t}"
      :
      : "r"(d), "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

// Bounded wait for the completion of phase `phase` of an mbarrier: false after
// 2^22 polls, or (with `abort` given) as soon as another thread of the CTA
// has raised the abort flag, so that one give-up ends every role's waits
// quickly.  A wait that gives up leaves its asynchronous operation in flight;
// rowinit_mma_kernel drains those before it frees tensor memory and exits.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, const volatile int *abort = nullptr) {
  for (int i = 0; i < (1 << 22); ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
    if (abort && (i & 255) == 255 && *abort) return false;
  }
  return false;
}

// Pack rows of a K-contiguous operand (count rows x K per lane, lane stride
// count x K) into limb tiles of `rows_per_tile` rows: tile (lane, block, step)
// at ((lane x blocks + block) x steps + step) x tile_bytes.
__global__ void __launch_bounds__(256) rowinit_pack_kernel(const uint32_t *src, uint64_t count, int K, int L,
                                                           int rows_per_tile, unsigned char *dst) {
  const int steps = (K + MK - 1) / MK;
  const uint64_t blocks = (count + rows_per_tile - 1) / rows_per_tile;
  const int limb_bytes = rows_per_tile * MK, tile_bytes = 4 * limb_bytes;
  const uint64_t total = uint64_t(L) * blocks * uint64_t(rows_per_tile) * uint64_t(steps);
  for (uint64_t w = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; w < total; w += uint64_t(gridDim.x) * blockDim.x) {
    const int ks = int(w % uint64_t(steps));
    uint64_t rest = w / uint64_t(steps);
    const int r = int(rest % uint64_t(rows_per_tile));
    rest /= uint64_t(rows_per_tile);
    const uint64_t blk = rest % blocks, l = rest / blocks;
    const uint64_t row = blk * uint64_t(rows_per_tile) + uint64_t(r);
    const uint32_t *rp = src + (l * count + row) * uint64_t(K);
    uint32_t v[MK];
#pragma unroll
    for (int k = 0; k < MK; ++k) v[k] = (row < count && ks * MK + k < K) ? rp[ks * MK + k] : 0u;
    unsigned char *tile = dst + ((l * blocks + blk) * uint64_t(steps) + uint64_t(ks)) * uint64_t(tile_bytes);
    const int roff = (r >> 3) * 256 + (r & 7) * 16;
#pragma unroll
    for (int limb = 0; limb < 4; ++limb) {
      const int sh = 8 * limb;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        uint32_t q4[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int k = c * 16 + q * 4;
          q4[q] = ((v[k] >> sh) & 0xffu) | (((v[k + 1] >> sh) & 0xffu) << 8) | (((v[k + 2] >> sh) & 0xffu) << 16) |
                  (((v[k + 3] >> sh) & 0xffu) << 24);
        }
        *reinterpret_cast<uint4 *>(tile + limb * limb_bytes + roff + c * 128) = make_uint4(q4[0], q4[1], q4[2], q4[3]);
      }
    }
  }
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// Item it of a product: its row tile, column tile and lane group.  Groups are
// innermost; row tiles run in bands of RBAND, a band sweeping every column tile.
__device__ __forceinline__ void mma_item(uint64_t it, int ngroups, uint64_t rblocks, uint64_t cblocks, uint64_t &rb,
                                         uint64_t &cb, int &grp) {
  grp = int(it % uint64_t(ngroups));
  const uint64_t t = it / uint64_t(ngroups);
  const uint64_t full = rblocks / RBAND, band = uint64_t(RBAND) * cblocks;
  if (t < full * band) {
    const uint64_t r = t % band;
    cb = r / RBAND;
    rb = (t / band) * RBAND + r % RBAND;
  } else {
    const uint64_t tail = rblocks - full * RBAND, r = t - full * band;
    cb = r / tail;
    rb = full * RBAND + r % tail;
  }
}

__global__ void __launch_bounds__(256, 1) rowinit_mma_kernel(Lanes ln, int K, uint64_t n, uint64_t C,
                                                             const unsigned char *Ap, const unsigned char *Bp,
                                                             const uint64_t *base, uint32_t *out,
                                                             unsigned int *err) {
  extern __shared__ __align__(128) unsigned char dsm[];
  __shared__ __align__(8) uint64_t full_bar[NST], empty_bar[NST], acc_full, acc_empty, drain_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  volatile int *abort_v = &abort_flag;
  uint32_t *stage_out = reinterpret_cast<uint32_t *>(dsm + kRingBytes);
  const int t = threadIdx.x, warp = t >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 0) {
    for (int i = 0; i < NST; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&full_bar[i])), "r"(1) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&empty_bar[i])), "r"(1) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&acc_full)), "r"(1) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&acc_empty)), "r"(128) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&drain_bar)), "r"(1) : "memory");
    abort_flag = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const int nks = (K + MK - 1) / MK;
  const int ngroups = ln.ngroups;
  const uint64_t rblocks = (n + MM - 1) / MM, cblocks = (C + MN - 1) / MN;
  const uint64_t items = rblocks * cblocks * uint64_t(ngroups);
  const uint64_t my_items = items > blockIdx.x ? (items - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  if (t == 0) {
    // Producer and MMA issuer.  The copy cursor (pk, pl, pks) runs up to
    // NST - 1 steps ahead of the MMAs; a lane's MMAs start once the epilogue
    // has read the previous lane's accumulators out of tensor memory.
    uint64_t pk = 0, prb = 0, pcb = 0;
    int pl = 0, pks = 0, pgrp = 0;
    if (my_items) mma_item(blockIdx.x, ngroups, rblocks, cblocks, prb, pcb, pgrp);
    uint64_t issued = 0, g = 0, lic = 0;
    auto issue_copy = [&]() -> bool {
      const int s = int(issued % NST);
      const uint64_t use = issued / NST;
      if (use > 0 && !mbar_wait(smem_addr(&empty_bar[s]), uint32_t((use - 1) & 1u), abort_v)) return false;
      const uint64_t lane = uint64_t(ln.grp_lane0[pgrp] + pl);
      const unsigned char *a = Ap + ((lane * rblocks + prb) * uint64_t(nks) + uint64_t(pks)) * uint64_t(A_TILE);
      const unsigned char *b = Bp + ((lane * cblocks + pcb) * uint64_t(nks) + uint64_t(pks)) * uint64_t(B_TILE);
      const uint32_t fb = smem_addr(&full_bar[s]);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(uint32_t(A_TILE + B_TILE)), "r"(fb)
                   : "memory");
      unsigned char *st = dsm + size_t(s) * (A_TILE + B_TILE);
      bulk_load(smem_addr(st), a, A_TILE, fb);
      bulk_load(smem_addr(st + A_TILE), b, B_TILE, fb);
      ++issued;
      if (++pks == nks) {
        pks = 0;
        if (++pl == ln.grp_n[pgrp]) {
          pl = 0;
          if (++pk < my_items) mma_item(blockIdx.x + pk * gridDim.x, ngroups, rblocks, cblocks, prb, pcb, pgrp);
        }
      }
      return true;
    };
    for (uint64_t k = 0; k < my_items && !*abort_v; ++k) {
      uint64_t rb, cb;
      int grp;
      mma_item(blockIdx.x + k * gridDim.x, ngroups, rblocks, cblocks, rb, cb, grp);
      for (int li = 0; li < ln.grp_n[grp] && !*abort_v; ++li, ++lic) {
        while (pk < my_items && issued < g + NST - 1) {
          if (!issue_copy()) {
            *abort_v = 1;
            break;
          }
        }
        if (*abort_v) break;
        if (lic > 0 && !mbar_wait(smem_addr(&acc_empty), uint32_t((lic - 1) & 1u), abort_v)) {
          *abort_v = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        for (int ks = 0; ks < nks; ++ks, ++g) {
          const int s = int(g % NST);
          if (!mbar_wait(smem_addr(&full_bar[s]), uint32_t((g / NST) & 1u), abort_v)) {
            *abort_v = 1;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const unsigned char *st = dsm + size_t(s) * (A_TILE + B_TILE);
          // The B tile's four limbs are one 256-row operand, so A limb i times
          // all of B is one N = 256 MMA whose column block j lands at
          // 64 (i + j), the accumulator of its shift.  The first step writes
          // each accumulator fresh once: limb 0 covers shifts 0..3, and limb
          // i >= 1 adds onto shifts i..i+2 and starts shift i + 3.
          const uint64_t dA = umma_desc(smem_addr(st)), dB = umma_desc(smem_addr(st + A_TILE));
          if (ks > 0) {
#pragma unroll
            for (int i = 0; i < 4; ++i) mma_i8(tmem + uint32_t(i * MN), dA + uint64_t(i * (A_LIMB >> 4)), dB, kIdescN256, 1u);
          } else {
            mma_i8(tmem, dA, dB, kIdescN256, 0u);
#pragma unroll
            for (int i = 1; i < 4; ++i) {
              const uint64_t da = dA + uint64_t(i * (A_LIMB >> 4));
              mma_i8(tmem + uint32_t(i * MN), da, dB, kIdescN192, 1u);
              mma_i8(tmem + uint32_t((i + 3) * MN), da, dB + uint64_t(3 * (B_LIMB >> 4)), kIdescI8, 0u);
            }
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_addr(&empty_bar[s]))
                       : "memory");
          // Refill the stage of step g - 1 (its MMAs were issued before these
          // ones) with step g + NST - 1 while this step's MMAs run.
          if (pk < my_items && issued == g + NST - 1 && !issue_copy()) {
            *abort_v = 1;
            break;
          }
        }
        if (*abort_v) break;
        // The lane's accumulators are complete once its MMAs are.
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&acc_full))
                     : "memory");
      }
    }
    if (*abort_v) {
      // Drain before the CTA frees tensor memory and its shared memory: a
      // commit to drain_bar arrives once every MMA this thread issued has
      // completed, and each bulk copy issued but never consumed (steps
      // g .. issued-1, one per ring stage at most) completes its stage's
      // full barrier.  Both waits are bounded; a drain that still gives up
      // leaves the error flag set all the same.
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&drain_bar))
                   : "memory");
      mbar_wait(smem_addr(&drain_bar), 0u);
      for (uint64_t c = g; c < issued; ++c) mbar_wait(smem_addr(&full_bar[c % NST]), uint32_t((c / NST) & 1u));
    }
  } else if (warp >= 4) {
    // Epilogue warps 4..7: warp w owns tensor-memory lanes (tile rows)
    // 32 (w - 4) .. + 31 and the same rows of the staging buffer, so only
    // the warp itself reads back what it parked there.  G_s < 4 K 255^2 <
    // 2^28 (K <= 1024), so sum_s G_s (2^(8s) mod p) < 7 x 2^60 fits 64 bits.
    const int quarter = warp - 4, lane_t = t & 31, row = quarter * 32 + lane_t;
    uint32_t *my_row = stage_out + size_t(row) * SROW;
    uint64_t lic = 0;
    for (uint64_t k = 0; k < my_items && !*abort_v; ++k) {
      uint64_t rb, cb;
      int grp;
      mma_item(blockIdx.x + k * gridDim.x, ngroups, rblocks, cblocks, rb, cb, grp);
      const int G = ln.grp_n[grp], lane0 = ln.grp_lane0[grp];
      const uint64_t gi_mine = rb * MM + uint64_t(row), j0 = cb * MN;
      const uint64_t my_base = gi_mine < n ? base[gi_mine] : 0;
      bool ok = true;
      for (int li = 0; li < G; ++li, ++lic) {
        if (!mbar_wait(smem_addr(&acc_full), uint32_t(lic & 1u), abort_v)) {
          *abort_v = 1;
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int l = lane0 + li;
        unsigned long long acc[MN];
#pragma unroll
        for (int q = 0; q < MN; ++q) acc[q] = 0;
#pragma unroll
        for (int c = 0; c < MN; c += 16) {
#pragma unroll
          for (int sft = 0; sft < 7; ++sft) {
            uint32_t gv[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];"
                : "=r"(gv[0]), "=r"(gv[1]), "=r"(gv[2]), "=r"(gv[3]), "=r"(gv[4]), "=r"(gv[5]), "=r"(gv[6]),
                  "=r"(gv[7]), "=r"(gv[8]), "=r"(gv[9]), "=r"(gv[10]), "=r"(gv[11]), "=r"(gv[12]), "=r"(gv[13]),
                  "=r"(gv[14]), "=r"(gv[15])
                : "r"(tmem + (uint32_t(quarter * 32) << 16) + uint32_t(sft * MN + c)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const uint32_t cs = ln.c8[l][sft];
#pragma unroll
            for (int q = 0; q < 16; ++q) acc[c + q] += (unsigned long long)gv[q] * cs;
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&acc_empty)) : "memory");
        const uint32_t p = ln.p[l];
        const unsigned long long m = ln.m[l];
#pragma unroll
        for (int q = 0; q < MN; ++q) my_row[q * 4 + li] = red64(acc[q], p, m);
      }
      if (!ok) break;
      __syncwarp();
      // Write the warp's 32 rows: row r holds states base[r] + j0 .. + 63,
      // each state's G lanes adjacent in the panel (G words from the group's
      // first lane, 4 G-byte aligned: panels start at multiples of their width).
      const uint32_t pw = uint32_t(ln.pw[lane0]);
      uint32_t *o = out + ln.off[lane0];
      for (int rr = 0; rr < 32; ++rr) {
        const uint64_t b0 = __shfl_sync(0xffffffffu, my_base, rr);
        if (rb * MM + uint64_t(quarter * 32 + rr) >= n) break;  // the same for the whole warp
        const uint32_t *src = stage_out + size_t(quarter * 32 + rr) * SROW;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int q = lane_t + 32 * h;
          if (j0 + uint64_t(q) >= C) continue;
          const uint4 v = *reinterpret_cast<const uint4 *>(src + q * 4);
          uint32_t *dst = o + (b0 + j0 + uint64_t(q)) * pw;
          if (G == 4) *reinterpret_cast<uint4 *>(dst) = v;
          else if (G == 2) *reinterpret_cast<uint2 *>(dst) = make_uint2(v.x, v.y);
          else *dst = v.x;
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  if (t == 0 && abort_flag) atomicExch(err, 1u);
}

struct RowInitDevice {
  RowInitPlan plan;
  AutDev aut{};
  std::vector<void *> allocs;
  // prefix levels (concatenated) and per-level offsets
  std::vector<size_t> lvl_off;  // prefixes before level k (size P + 1)
  int32_t *parent = nullptr, *row = nullptr;
  uint8_t *sym = nullptr, *height = nullptr;
  uint64_t *base_hr = nullptr;  // level P bases by (height, row)
  std::vector<uint64_t> base_hoff;
  ~RowInitDevice() {
    for (void *p : allocs) cudaFree(p);
  }
};

template <typename T>
cudaError_t upload(RowInitDevice &d, const std::vector<T> &h, T **out) {
  *out = nullptr;
  const size_t bytes = std::max<size_t>(1, h.size()) * sizeof(T);
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(out), bytes);
  if (e != cudaSuccess) return e;
  d.allocs.push_back(*out);
  if (h.empty()) return cudaSuccess;
  return cudaMemcpy(*out, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
}

cudaError_t build_device(int W, int rows, int cap, std::unique_ptr<RowInitDevice> &out) {
  auto d = std::make_unique<RowInitDevice>();
  d->plan = plan_row_init(W, rows, cap);
  const RowInitPlan &pl = d->plan;
  const RowAutomaton &a = row_automaton(rows);
  AutDev &ad = d->aut;
  ad.n = a.nstates;
  int acc = 0;
  for (int h = 0; h < kH; ++h) {
    ad.K[h] = h <= rows ? a.per_height[size_t(h)] : 0;
    ad.hoff[h] = acc;
    acc += ad.K[h];
  }
  std::vector<int> gid(size_t(std::max(acc, 1)), 0);
  for (int s = 0; s < a.nstates; ++s) gid[size_t(ad.hoff[a.height[size_t(s)]] + a.index[size_t(s)])] = s;
  std::vector<int> first_off(4, 0), first_to;
  std::vector<uint32_t> first_w;
  for (int s = 0; s < 3; ++s) {
    for (const AutTrans &t : a.first[s]) {
      first_to.push_back(a.index[size_t(t.to)]);
      first_w.push_back(t.weight);
    }
    first_off[size_t(s) + 1] = int(first_to.size());
  }
  std::vector<int> fwd_off(size_t(3) * (a.nstates + 1), 0), fwd_from, bwd_off(size_t(3) * (a.nstates + 1), 0), bwd_to;
  std::vector<uint32_t> fwd_w, bwd_w, last_w(size_t(3) * a.nstates, 0);
  for (int s = 0; s < 3; ++s) {
    std::vector<std::vector<std::pair<int, uint32_t>>> in(size_t(a.nstates)), outv(size_t(a.nstates));
    for (const AutTrans &t : a.inner[s]) {
      in[size_t(t.to)].push_back({a.index[size_t(t.from)], t.weight});
      outv[size_t(t.from)].push_back({a.index[size_t(t.to)], t.weight});
    }
    int *fo = fwd_off.data() + size_t(s) * (a.nstates + 1), *bo = bwd_off.data() + size_t(s) * (a.nstates + 1);
    fo[0] = int(fwd_from.size());
    bo[0] = int(bwd_to.size());
    for (int q = 0; q < a.nstates; ++q) {
      for (auto &e : in[size_t(q)]) {
        fwd_from.push_back(e.first);
        fwd_w.push_back(e.second);
      }
      fo[q + 1] = int(fwd_from.size());
      for (auto &e : outv[size_t(q)]) {
        bwd_to.push_back(e.first);
        bwd_w.push_back(e.second);
      }
      bo[q + 1] = int(bwd_to.size());
    }
    for (const AutTrans &t : a.last[s]) last_w[size_t(s) * a.nstates + size_t(t.from)] += t.weight;
  }
  cudaError_t e;
#define UP(vec, ptr)                                                      \
  if ((e = upload(*d, vec, &ptr)) != cudaSuccess) return e;
  int *p_gid, *p_fo, *p_ft, *p_fwo, *p_fwf, *p_bwo, *p_bwt;
  uint32_t *p_fw, *p_fww, *p_bww, *p_lw;
  UP(gid, p_gid) UP(first_off, p_fo) UP(first_to, p_ft) UP(first_w, p_fw) UP(fwd_off, p_fwo) UP(fwd_from, p_fwf)
  UP(fwd_w, p_fww) UP(bwd_off, p_bwo) UP(bwd_to, p_bwt) UP(bwd_w, p_bww) UP(last_w, p_lw)
  ad.gid = p_gid;
  ad.first_off = p_fo;
  ad.first_to = p_ft;
  ad.first_w = p_fw;
  ad.fwd_off = p_fwo;
  ad.fwd_from = p_fwf;
  ad.fwd_w = p_fww;
  ad.bwd_off = p_bwo;
  ad.bwd_to = p_bwt;
  ad.bwd_w = p_bww;
  ad.last_w = p_lw;
  // Prefix levels.
  std::vector<int32_t> par, rw;
  std::vector<uint8_t> sy, hh;
  d->lvl_off.assign(1, 0);
  for (int k = 0; k < pl.P; ++k) {
    par.insert(par.end(), pl.parent[size_t(k)].begin(), pl.parent[size_t(k)].end());
    rw.insert(rw.end(), pl.row[size_t(k)].begin(), pl.row[size_t(k)].end());
    sy.insert(sy.end(), pl.sym[size_t(k)].begin(), pl.sym[size_t(k)].end());
    hh.insert(hh.end(), pl.height[size_t(k)].begin(), pl.height[size_t(k)].end());
    d->lvl_off.push_back(par.size());
  }
  UP(par, d->parent) UP(rw, d->row) UP(sy, d->sym) UP(hh, d->height)
  // Level-P bases by (height, row).
  const auto &htop = pl.height[size_t(pl.P - 1)];
  const auto &rtop = pl.row[size_t(pl.P - 1)];
  d->base_hoff.assign(kH + 1, 0);
  for (int h = 0; h < kH; ++h)
    d->base_hoff[size_t(h) + 1] = d->base_hoff[size_t(h)] + (h <= rows ? pl.rows_of[size_t(pl.P - 1)][size_t(h)] : 0);
  std::vector<uint64_t> bhr(size_t(d->base_hoff[kH]), 0);
  for (size_t i = 0; i < htop.size(); ++i) bhr[size_t(d->base_hoff[htop[i]]) + size_t(rtop[i])] = pl.base[i];
  UP(bhr, d->base_hr)
#undef UP
  if ((e = cudaFuncSetAttribute(rowinit_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kMmaSmem))) !=
      cudaSuccess)
    return e;
  out = std::move(d);
  return cudaSuccess;
}

std::mutex g_mu;
std::map<std::tuple<int, int, int, int>, std::unique_ptr<RowInitDevice>> g_cache;  // (device, W, rows, cap)

LevelArgs level_args(const std::vector<uint64_t> &cnt, const int *K, int hmax, int L) {
  LevelArgs a{};
  uint64_t off = 0;
  for (int h = 0; h < kH; ++h) {
    a.cnt[h] = h <= hmax && h < int(cnt.size()) ? cnt[size_t(h)] : 0;
    a.base[h] = off;
    off += a.cnt[h] * uint64_t(K[h]) * uint64_t(L);
  }
  return a;
}

}  // namespace

cudaError_t prepare_row_init(int W, int rows, int cap) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_mu);
  auto key = std::make_tuple(dev, W, rows, cap);
  if (g_cache.count(key)) return cudaSuccess;
  std::unique_ptr<RowInitDevice> d;
  if ((e = build_device(W, rows, cap, d)) != cudaSuccess) return e;
  g_cache.emplace(key, std::move(d));
  return cudaSuccess;
}

int auto_row_init_rows(int W) { return W >= 18 ? 7 : (W >= 14 ? 6 : 0); }

// Scratch words per lane and table bytes of a fill plan, computed once per
// (W, rows, cap): planning large widths takes a moment on the host.
static std::pair<uint64_t, uint64_t> row_init_sizes(int W, int rows, int cap) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int>, std::pair<uint64_t, uint64_t>> sizes;
  std::lock_guard<std::mutex> lk(mu);
  auto key = std::make_tuple(W, rows, cap);
  auto it = sizes.find(key);
  if (it == sizes.end()) {
    const RowInitPlan pl = plan_row_init(W, rows, cap);
    it = sizes.emplace(key, std::make_pair(row_init_scratch_words(pl), row_init_table_bytes(pl))).first;
  }
  return it->second;
}

uint64_t row_init_scratch(int W, int rows, int cap) { return row_init_sizes(W, rows, cap).first; }

uint64_t row_init_tables(int W, int rows, int cap) { return row_init_sizes(W, rows, cap).second; }

cudaError_t enqueue_row_init(int W, int rows, int cap, int L, const uint32_t *mods, uint32_t *main,
                             uint32_t *scratch, uint64_t scratch_words, bool tensor, unsigned int *err,
                             cudaStream_t s, uint64_t *launches) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  RowInitDevice *d = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_cache.find(std::make_tuple(dev, W, rows, cap));
    if (it == g_cache.end()) return cudaErrorNotReady;  // prepare_row_init first (outside capture)
    d = it->second.get();
  }
  const RowInitPlan &pl = d->plan;
  if (L < 1 || L > 16 || (tensor && !err)) return cudaErrorInvalidValue;
  if (row_init_scratch_words(pl) * uint64_t(L) > scratch_words) return cudaErrorInvalidValue;
  Lanes ln{};
  for (int l = 0; l < L;) {
    const int pw = (L - l >= 8) ? 8 : (L - l >= 4) ? 4 : (L - l >= 2) ? 2 : 1;
    for (int i = 0; i < pw; ++i) {
      ln.off[l + i] = uint64_t(l) * pl.states + uint64_t(i);
      ln.pw[l + i] = pw;
    }
    for (int g0 = 0; g0 < pw; g0 += 4) {
      ln.grp_lane0[ln.ngroups] = l + g0;
      ln.grp_n[ln.ngroups] = std::min(4, pw - g0);
      ++ln.ngroups;
    }
    l += pw;
  }
  for (int l = 0; l < L; ++l) {
    ln.p[l] = mods[l];
    ln.m[l] = ~0ull / mods[l];
    uint64_t c = 1 % mods[l];
    for (int sft = 0; sft < 7; ++sft) {
      ln.c8[l][sft] = uint32_t(c);
      c = (c << 8) % mods[l];
    }
  }
  uint64_t pre_words = 0, suf_words = 0;
  for (int k = 0; k < pl.P; ++k) {
    uint64_t w = 0;
    for (int h = 0; h <= pl.hmax; ++h) w += pl.rows_of[size_t(k)][size_t(h)] * uint64_t(pl.K[size_t(h)]);
    pre_words = std::max(pre_words, w * uint64_t(L));
  }
  for (int k = 1; k <= pl.S; ++k) {
    uint64_t w = 0;
    for (int g = 0; g <= pl.hmax; ++g) w += pl.C[size_t(k)][size_t(g)] * uint64_t(pl.K[size_t(g)]);
    suf_words = std::max(suf_words, w * uint64_t(L));
  }
  pre_words = (pre_words + 3) & ~uint64_t(3);
  suf_words = (suf_words + 3) & ~uint64_t(3);
  uint32_t *pre[2] = {scratch, scratch + pre_words};
  uint32_t *suf[2] = {scratch + 2 * pre_words, scratch + 2 * pre_words + suf_words};
  if ((e = cudaMemsetAsync(main, 0, size_t(pl.states) * L * 4, s)) != cudaSuccess) return e;
  const int blocks = device_sm_count() * 8;
  uint64_t n = 0;
  // Prefix levels 1..P.
  LevelArgs prevA{};
  for (int k = 1; k <= pl.P; ++k) {
    const LevelArgs cur = level_args(pl.rows_of[size_t(k - 1)], d->aut.K, pl.hmax, L);
    const size_t o = d->lvl_off[size_t(k - 1)], po = k > 1 ? d->lvl_off[size_t(k - 2)] : 0;
    const int np = int(d->lvl_off[size_t(k)] - o);
    rowinit_prefix_kernel<<<blocks, 256, 0, s>>>(d->aut, ln, L, k == 1, np, d->parent + o, d->sym + o, d->height + o,
                                                 d->row + o, d->height + po, d->row + po, cur, prevA,
                                                 pre[(k + 1) & 1], pre[k & 1]);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    ++n;
    prevA = cur;
  }
  // Suffix levels 1..S.
  LevelArgs prevU{};
  for (int k = 1; k <= pl.S; ++k) {
    std::vector<uint64_t> cnt(pl.C[size_t(k)].begin(), pl.C[size_t(k)].end());
    const LevelArgs cur = level_args(cnt, d->aut.K, pl.hmax, L);
    SufCounts sc{};
    for (int g = 0; g < kH; ++g) {
      sc.cur[g] = g <= pl.hmax ? pl.C[size_t(k)][size_t(g)] : 0;
      sc.prev[g] = (k > 1 && g <= pl.hmax) ? pl.C[size_t(k - 1)][size_t(g)] : 0;
    }
    rowinit_suffix_kernel<<<blocks, 256, 0, s>>>(d->aut, ln, L, k == 1, pl.hmax, sc, cur, prevU, suf[(k + 1) & 1],
                                                 suf[k & 1]);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    ++n;
    prevU = cur;
  }
  // Products, one launch per end height.
  const uint32_t *V = pre[pl.P & 1], *U = suf[pl.S & 1];
  for (int h = 0; h <= pl.hmax; ++h) {
    const uint64_t rows_h = prevA.cnt[h], cols = prevU.cnt[h];
    const int K = d->aut.K[h];
    if (!rows_h || !cols || !K) continue;
    if (tensor && K <= 1024) {
      // Packed limb tiles after the level buffers (16-byte aligned).
      unsigned char *ap = reinterpret_cast<unsigned char *>(scratch + 2 * pre_words + 2 * suf_words);
      const uint64_t nks = uint64_t(K + MK - 1) / MK, rblocks = (rows_h + MM - 1) / MM, cblocks = (cols + MN - 1) / MN;
      unsigned char *bp = ap + uint64_t(L) * rblocks * nks * A_TILE;
      const int pblocks = device_sm_count() * 8;
      rowinit_pack_kernel<<<pblocks, 256, 0, s>>>(V + prevA.base[h], rows_h, K, L, MM, ap);
      rowinit_pack_kernel<<<pblocks, 256, 0, s>>>(U + prevU.base[h], cols, K, L, MN, bp);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      n += 2;
      const uint64_t items = rblocks * cblocks * uint64_t(ln.ngroups);
      const uint64_t grid = std::min<uint64_t>(items, uint64_t(device_sm_count()));
      rowinit_mma_kernel<<<unsigned(grid), 256, kMmaSmem, s>>>(ln, K, rows_h, cols, ap, bp,
                                                                d->base_hr + d->base_hoff[size_t(h)], main, err);
    } else {
      const uint64_t tiles = ((rows_h + TM - 1) / TM) * ((cols + TN - 1) / TN);
      rowinit_product_kernel<<<unsigned(tiles), 256, 0, s>>>(ln, L, K, rows_h, cols, V + prevA.base[h],
                                                             U + prevU.base[h],
                                                             d->base_hr + d->base_hoff[size_t(h)], main);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    ++n;
  }
  if (launches) *launches += n;
  return cudaSuccess;
}

}  // namespace fdp
