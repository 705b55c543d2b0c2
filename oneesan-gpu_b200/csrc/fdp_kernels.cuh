// sm_100a kernels of the frontier DP: the per-cell transition (pull form, in
// place, no atomics), the row-0 initialiser and the first-row dot product.
// The per-item arithmetic lives in fdp_item.cuh.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fdp_item.cuh"

namespace fdp {

template <typename Idx>
__device__ __forceinline__ void load_cell_smem(CellSmem<Idx> &sm, const WidthTables<Idx> *t, int W, int p) {
  const int nthr = blockDim.x, tid = threadIdx.x;
  for (int i = tid; i < (FDP_MAXW + 1) * FDP_HS; i += nthr) sm.H[i / FDP_HS][i % FDP_HS] = t->H[i / FDP_HS][i % FDP_HS];
  // Only blocked positions p..W-2 are walked by the prefix decode.
  const int rows = W - 1 - p;
  for (int i = tid; i < rows * FDP_HS; i += nthr) {
    const int pos = p + i / FDP_HS, h = i % FDP_HS;
    sm.S[pos][h] = t->S[pos][h];
  }
  for (int i = tid; i < FDP_HS * PR_COUNT; i += nthr) sm.OFF[i / PR_COUNT][i % PR_COUNT] = t->OFF[p][i / PR_COUNT][i % PR_COUNT];
}

// Dynamic shared memory of the cell kernel: the width tables, the
// closure-candidate slots (slot i of thread t at cand[i * blockDim + t],
// cand_slots(W) slots), then (grouped small-p launches) one head store per
// warp: rec_items states per lane (compact = 1) or the carry-over queues
// (compact = 2).
template <typename Idx, int K>
FDP_HD constexpr size_t cell_recs_offset(int block, int W) {
  return (sizeof(CellSmem<Idx>) + (stages_candidates<K>() ? size_t(cand_slots(W)) * block * sizeof(Idx) : 0) +
          15) &
         ~size_t(15);
}

template <typename Idx>
FDP_HD constexpr size_t cell_recs_per_warp(int compact, int rec_items) {
  return compact == 2 ? carry_rec_bytes<Idx>()
                      : (compact == 1 ? size_t(32 * rec_items) * head_rec_entry_bytes<Idx>() : size_t(0));
}

template <typename Idx, int K>
FDP_HD constexpr size_t cell_smem_bytes(int block, int W, int compact, int rec_items) {
  return cell_recs_offset<Idx, K>(block, W) + size_t(block / 32) * cell_recs_per_warp<Idx>(compact, rec_items);
}

// Resident CTAs of 256 threads per SM the cell kernels are compiled for
// unless a lane count has its own budget below (64 registers per thread).
#ifndef FDP_CELL_MIN_BLOCKS
#define FDP_CELL_MIN_BLOCKS 4
#endif

template <typename Idx, int K, bool GROUPED>
__device__ __forceinline__ void cell_body(const CellArgs &a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CellSmem<Idx> &sm = *reinterpret_cast<CellSmem<Idx> *>(smem_raw);
  Idx *cand = reinterpret_cast<Idx *>(smem_raw + sizeof(CellSmem<Idx>));
  load_cell_smem<Idx>(sm, reinterpret_cast<const WidthTables<Idx> *>(a.tables), a.W, a.p);
  __syncthreads();
  // Each warp takes chunks of 32 * lane_items consecutive blocked indices;
  // lane l handles indices l, l + 32, ... of its chunk, so every access of a
  // warp still covers 32 consecutive states.  With share_prefix the top
  // symbols common to the whole chunk are decoded once (a warp-uniform walk on
  // broadcast shared-memory reads) instead of once per index.
  const Idx n = Idx(a.items);
  const Idx chunk = Idx(32) * Idx(a.lane_items > 0 ? a.lane_items : 1);
  const Idx wpb = Idx(blockDim.x >> 5);
  const Idx step = Idx(gridDim.x) * wpb * chunk;
  const Idx lane = Idx(threadIdx.x & 31);
  // Compacted (cells where a warp's items mix centre types, p small): the
  // heads of a chunk are decoded first and stored split by type, c = R/L from
  // the front and c = N from the back, so each update runs on whole warps
  // instead of two half-empty branches.  Any order of items within a cell is
  // valid: no item reads or writes a word another item writes.
  const int compact = !GROUPED ? 0 : (a.compact == 2 ? 2 : (a.compact && a.lane_items <= FDP_REC_MAX_ITEMS ? 1 : 0));
  unsigned char *const recs = smem_raw + cell_recs_offset<Idx, K>(blockDim.x, a.W) +
                              size_t(threadIdx.x >> 5) * cell_recs_per_warp<Idx>(compact, a.lane_items);
  const HeadRecs<Idx> rec{recs, int(chunk)};
  const CarryRecs<Idx> cr{recs};
  int qx = 0, qn = 0;  // carry-over queue depths (warp-uniform)
  const unsigned below = (1u << (threadIdx.x & 31)) - 1u;
  for (Idx jb = (Idx(blockIdx.x) * wpb + Idx(threadIdx.x >> 5)) * chunk; jb < n; jb += step) {
    const Idx jl = (n - jb > chunk) ? jb + chunk - 1 : n - 1;
    const Prefix<Idx> pf = a.share_prefix ? shared_prefix<Idx>(a, sm, jb, jl) : empty_prefix<Idx>(a);
    const Idx span = jl - jb;
    if (compact == 0) {
      for (Idx j = jb + lane; j <= jl; j += 32) cell_item<Idx, K>(a, sm, j, pf, cand + threadIdx.x, int(blockDim.x));
    } else if (compact == 1) {
      const int last = int(chunk) - 1;
      int nx = 0, nn = 0;
      for (int i = 0; i < a.lane_items; ++i) {
        const Idx o = lane + Idx(32 * i);
        const bool valid = o <= span;
        Head<Idx> hd{};
        if (valid) hd = decode_head<Idx>(a, sm, jb + o, pf);
        const bool isx = valid && hd.c != 0, isn = valid && hd.c == 0;
        const unsigned bx = __ballot_sync(0xffffffffu, isx), bn = __ballot_sync(0xffffffffu, isn);
        if (isx) rec.put(nx + __popc(bx & below), hd);
        if (isn) rec.put(last - (nn + __popc(bn & below)), hd);
        nx += __popc(bx);
        nn += __popc(bn);
      }
      __syncwarp();
      for (int k = int(lane); k < nx; k += 32) item_x<Idx, K>(a, sm, rec.get(k));
      for (int k = int(lane); k < nn; k += 32)
        item_n<Idx, K>(a, sm, rec.get(last - k), cand + threadIdx.x, int(blockDim.x));
      __syncwarp();
    } else {
      // Carry-over: push one head per lane, then update 32 items of a type as
      // soon as 32 wait; the rest stay queued for the next chunk.  Each queue
      // holds at most 31 + 32 entries.
      for (int i = 0; i < a.lane_items; ++i) {
        const Idx o = lane + Idx(32 * i);
        const bool valid = o <= span;
        Head<Idx> hd{};
        if (valid) hd = decode_head<Idx>(a, sm, jb + o, pf);
        const bool isx = valid && hd.c != 0, isn = valid && hd.c == 0;
        const unsigned bx = __ballot_sync(0xffffffffu, isx), bn = __ballot_sync(0xffffffffu, isn);
        if (isx) {
          Idx ia, ib;
          x_words<Idx>(sm, hd, ia, ib);
          cr.put_x(qx + __popc(bx & below), ia, ib, hd.j);
        }
        if (isn) cr.put_n(qn + __popc(bn & below), hd);
        qx += __popc(bx);
        qn += __popc(bn);
        __syncwarp();
        if (qx >= 32) {
          qx -= 32;
          const int k = qx + int(lane);
          apply_x<Idx, K>(a, cr.f(0)[k], cr.f(1)[k], cr.f(2)[k]);
        }
        if (qn >= 32) {
          qn -= 32;
          item_n<Idx, K>(a, sm, cr.get_n(qn + int(lane)), cand + threadIdx.x, int(blockDim.x));
        }
        __syncwarp();
      }
    }
    if (n - jb <= step) break;  // the next chunk start would be past n (and may wrap)
  }
  // Whatever the carry-over queues still hold.
  if (int(lane) < qx) apply_x<Idx, K>(a, cr.f(0)[lane], cr.f(1)[lane], cr.f(2)[lane]);
  if (int(lane) < qn) item_n<Idx, K>(a, sm, cr.get_n(int(lane)), cand + threadIdx.x, int(blockDim.x));
}

// Resident CTAs of 256 threads per SM each variant is compiled for (the
// register budget per thread is 65536 / (256 x this)): narrow lane counts need
// fewer registers per item, so more warps keep loads in flight.  Measured at
// n = 22: the streaming cells of one lane 136 -> 109 ms per row at 6 CTAs (40
// registers), 2 and 4 lanes gain there too; the grouped cells of 2-4 lanes
// gain 3 % at 5 CTAs, those of one lane do not; 6 and 8 lanes spill and run
// 2-7 % slower at 5 or 6, so lane counts above 4 stay at 4.
template <int K>
constexpr int group_min_blocks() { return (K >= 2 && K <= 4) ? 5 : FDP_CELL_MIN_BLOCKS; }
template <int K>
constexpr int stream_min_blocks() { return K <= 4 ? 6 : FDP_CELL_MIN_BLOCKS; }

// The cell kernel of the cells whose items are grouped by centre type (small
// p) and the one of the cells that stream them in index order (the rest):
// the same body, compiled apart so that each gets its own register budget.
template <typename Idx, int K>
__global__ void __launch_bounds__(256, group_min_blocks<K>()) cell_kernel(const CellArgs a) {
  cell_body<Idx, K, true>(a);
}

template <typename Idx, int K>
__global__ void __launch_bounds__(256, stream_min_blocks<K>()) cell_stream_kernel(const CellArgs a) {
  cell_body<Idx, K, false>(a);
}

template <typename Idx, int K>
__global__ void __launch_bounds__(256) first_row_init_kernel(const FirstRowArgs a) {
  __shared__ Idx sH[FDP_MAXW + 1][FDP_HT];
  const WidthTables<Idx> *t = reinterpret_cast<const WidthTables<Idx> *>(a.tables);
  for (int i = threadIdx.x; i < (FDP_MAXW + 1) * FDP_HT; i += blockDim.x) (&sH[0][0])[i] = (&t->H[0][0])[i];
  __syncthreads();
  const uint64_t total = 1ull << (a.W - 1);
  uint32_t one[K];
#pragma unroll
  for (int i = 0; i < K; ++i) one[i] = 1u;
  for (uint64_t mask = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; mask < total;
       mask += uint64_t(gridDim.x) * blockDim.x) {
    const Idx rk = rank_dev<Idx>(first_row_state_dev(mask, a.W), a.W, sH);
    st_lanes<K>(a.main, a.mstates, size_t(rk), one);
  }
}

template <typename Idx, int K>
__global__ void __launch_bounds__(256) first_row_dot_kernel(const FirstRowArgs a) {
  __shared__ Idx sH[FDP_MAXW + 1][FDP_HT];
  __shared__ unsigned long long red[8][K];
  const WidthTables<Idx> *t = reinterpret_cast<const WidthTables<Idx> *>(a.tables);
  for (int i = threadIdx.x; i < (FDP_MAXW + 1) * FDP_HT; i += blockDim.x) (&sH[0][0])[i] = (&t->H[0][0])[i];
  __syncthreads();
  const uint64_t total = 1ull << (a.W - 1);
  unsigned long long acc[K];
#pragma unroll
  for (int i = 0; i < K; ++i) acc[i] = 0;
  for (uint64_t mask = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; mask < total;
       mask += uint64_t(gridDim.x) * blockDim.x) {
    const Idx rk = rank_dev<Idx>(first_row_state_dev(mask, a.W), a.W, sH);
    uint32_t v[K];
    ld_lanes<K>(a.main, a.mstates, size_t(rk), v);
#pragma unroll
    for (int i = 0; i < K; ++i) acc[i] += v[i];
  }
  // Exact 64-bit sums: at most 2^27 terms below 2^32 each.
#pragma unroll
  for (int i = 0; i < K; ++i) {
    unsigned long long v = acc[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][i] = v;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    unsigned long long v = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) v += red[w][threadIdx.x];
    atomicAdd(a.acc + threadIdx.x, v);
  }
}

// residue[k] = acc[k] mod p_k
__global__ void finalize_residues_kernel(const unsigned long long *acc, uint32_t *out, FirstRowArgs a, int k);

}  // namespace fdp
