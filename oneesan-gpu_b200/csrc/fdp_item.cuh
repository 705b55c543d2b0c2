// Per-item logic of the frontier-DP kernels (host+device so the host test
// harness and the sm_100a kernels share one definition).
//
// Per-cell operator (the semantics of src/common/gridfp_transition.hpp:113-146
// as driven by tests/groupbatch_operator_test.cu:127-146 of the reference):
//   main'  = main + sum over included main->main moves + blocked_exclude(blocked)
//   block' = sum over included main->blocked moves
// Work decomposition (this build's own): one work item per blocked index j at
// cell p.  Decoding j yields the high prefix (base `bm` in main, end height h),
// the centre symbol c at p-1 and the low rank r.  The item owns
//   c = N : main NN, main LR, block j     (reads RL and the LL/RR closure sources)
//   c = R : main NR, block j              (reads RN)
//   c = L : main NL, block j              (reads LN)
// and at p = 1 also main RN (c = R).  No two items write the same word and no
// item reads a word another item writes, so the update is race-free in place
// and needs no scratch: 4(M+D) bytes of state per modulus, nothing else.
//
// Moduli: K residues per state are interleaved, word index = state*K + k, so
// one decoded index serves K moduli with one contiguous K*4-byte access.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fdp_core.cuh"

namespace fdp {

struct CellArgs {
  const void *tables;  // WidthTables<Idx> in device memory
  uint32_t *main;      // [M][K]
  uint32_t *blk;       // [D][K]
  uint64_t items;      // D = blocked states
  uint32_t mod[16];
  int W, p;
  int blk_in_zero;     // blocked input known to be zero (first cell of a row sweep)
  int blk_out_p1;      // at p = 1 store the (all-zero) blocked output
};

struct FirstRowArgs {
  const void *tables;
  uint32_t *main;                 // [M][K]
  unsigned long long *acc;        // [K] 64-bit accumulators (dot product)
  uint32_t mod[16];
  int W;
};

// ---- K-wide loads / stores on the interleaved layout -----------------------
template <int K>
FDP_HD void ldk(const uint32_t *p, uint32_t (&x)[K]) {
  if constexpr (K % 4 == 0) {
#pragma unroll
    for (int i = 0; i < K / 4; ++i) {
      uint4 t = reinterpret_cast<const uint4 *>(p)[i];
      x[4 * i] = t.x; x[4 * i + 1] = t.y; x[4 * i + 2] = t.z; x[4 * i + 3] = t.w;
    }
  } else if constexpr (K % 2 == 0) {
#pragma unroll
    for (int i = 0; i < K / 2; ++i) {
      uint2 t = reinterpret_cast<const uint2 *>(p)[i];
      x[2 * i] = t.x; x[2 * i + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < K; ++i) x[i] = p[i];
  }
}

template <int K>
FDP_HD void stk(uint32_t *p, const uint32_t (&x)[K]) {
  if constexpr (K % 4 == 0) {
#pragma unroll
    for (int i = 0; i < K / 4; ++i)
      reinterpret_cast<uint4 *>(p)[i] = make_uint4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3]);
  } else if constexpr (K % 2 == 0) {
#pragma unroll
    for (int i = 0; i < K / 2; ++i) reinterpret_cast<uint2 *>(p)[i] = make_uint2(x[2 * i], x[2 * i + 1]);
  } else {
#pragma unroll
    for (int i = 0; i < K; ++i) p[i] = x[i];
  }
}

template <int K>
FDP_HD void acc_from(const uint32_t *p, uint32_t (&acc)[K], const uint32_t *mod) {
  uint32_t v[K];
  ldk<K>(p, v);
#pragma unroll
  for (int i = 0; i < K; ++i) acc[i] = add_mod(acc[i], v[i], mod[i]);
}

// ---- shared-memory copies of the width tables ------------------------------
template <typename Idx>
struct CellSmem {
  StepT<Idx> S[FDP_MAXW][FDP_HT];
  Idx H[FDP_MAXW + 1][FDP_HT];
  Idx OFF[FDP_HT][PR_COUNT];
};

// ---- the cell kernel --------------------------------------------------------
template <typename Idx, int K>
FDP_HD void cell_item(const CellArgs &a, const CellSmem<Idx> &sm, const Idx j) {
  const int W = a.W, p = a.p;
  // Decode the blocked prefix (blocked positions W-2..p) top-down.
  Idx r = j, bm = 0;
  int h = 1;
  uint64_t hw = 0;  // high symbols at their main positions W-1..p+1
  for (int pos = W - 2; pos >= p; --pos) {
    const StepT<Idx> s = sm.S[pos][h];
    if (r >= s.t1) {
      if (r >= s.t2) {
        r -= s.t2; bm += s.cL; hw |= uint64_t(SYM_L) << (2 * (pos + 1)); ++h;
      } else {
        r -= s.t1; bm += s.cR; hw |= uint64_t(SYM_R) << (2 * (pos + 1)); --h;
      }
    }
  }
  // Centre symbol at blocked position p-1 and the low rank r.
  int c = 0;
  {
    const Idx bN = sm.H[p - 1][h];
    if (r >= bN) {
      r -= bN;
      const Idx bR = h > 0 ? sm.H[p - 1][h - 1] : Idx(0);
      if (r < bR) c = 1;
      else { r -= bR; c = 2; }
    }
  }
  const Idx *off = sm.OFF[h];
  uint32_t *const Mn = a.main;
  uint32_t *const Bk = a.blk;
  const size_t jK = size_t(j) * K;
  const uint32_t *mod = a.mod;

  if (c != 0) {
    // c = R: NR' = NR + RN + B, B' = NR ;  c = L: NL' = NL + LN + B, B' = NL.
    // At p = 1 (only c = R reaches here): RN' = RN + NR as well.
    const Idx i1 = bm + off[c == 1 ? PR_NR : PR_NL] + r;
    const Idx i2 = bm + off[c == 1 ? PR_RN : PR_LN] + r;
    uint32_t x[K], y[K], z[K];
    ldk<K>(Mn + size_t(i1) * K, x);
    ldk<K>(Mn + size_t(i2) * K, y);
#pragma unroll
    for (int i = 0; i < K; ++i) z[i] = add_mod(x[i], y[i], mod[i]);
    if (!a.blk_in_zero) {
      uint32_t b[K];
      ldk<K>(Bk + jK, b);
#pragma unroll
      for (int i = 0; i < K; ++i) z[i] = add_mod(z[i], b[i], mod[i]);
    }
    stk<K>(Mn + size_t(i1) * K, z);
    if (p >= 2) {
      stk<K>(Bk + jK, x);
    } else {
#pragma unroll
      for (int i = 0; i < K; ++i) z[i] = add_mod(y[i], x[i], mod[i]);
      stk<K>(Mn + size_t(i2) * K, z);
      if (a.blk_out_p1) {
#pragma unroll
        for (int i = 0; i < K; ++i) z[i] = 0;
        stk<K>(Bk + jK, z);
      }
    }
    return;
  }

  // c = N: NN' = NN + B, LR' = LR + NN, B' = RL + closures (p >= 2);
  //        at p = 1: NN' = NN + B + RR closures, LR' = LR + NN.
  const Idx iNN = bm + off[PR_NN] + r;
  const Idx iLR = bm + off[PR_LR] + r;
  uint32_t x[K], acc[K];
  ldk<K>(Mn + size_t(iNN) * K, x);
  {
    uint32_t y[K];
    ldk<K>(Mn + size_t(iLR) * K, y);
#pragma unroll
    for (int i = 0; i < K; ++i) y[i] = add_mod(y[i], x[i], mod[i]);
    stk<K>(Mn + size_t(iLR) * K, y);
  }
  if (!a.blk_in_zero) {
    uint32_t b[K];
    ldk<K>(Bk + jK, b);
#pragma unroll
    for (int i = 0; i < K; ++i) x[i] = add_mod(x[i], b[i], mod[i]);
  }
#pragma unroll
  for (int i = 0; i < K; ++i) acc[i] = 0;
  if (p >= 2) {
    stk<K>(Mn + size_t(iNN) * K, x);
    if (h > 0) ldk<K>(Mn + size_t(bm + off[PR_RL] + r) * K, acc);
    // LL closures: every L at depth 1 of the low word, flipped to R, is a
    // predecessor with pair LL (RV.hpp:49-69 enumerates the same set).  Its
    // rank from height h+2 equals the +2-shifted prefix rank, plus H[pos][hb+2]
    // for the R, plus the unchanged remainder below.
    if (p >= 3) {
      const Idx baseLL = bm + off[PR_LL];
      Idx rem = r, pre2 = 0;
      int hb = h, depth = 1;
      for (int pos = p - 2; pos >= 0 && depth > 0; --pos) {
        const Idx z0 = sm.H[pos][hb];
        if (rem < z0) {
          // N: no contribution at either height
          continue;
        }
        rem -= z0;
        const Idx z1 = hb > 0 ? sm.H[pos][hb - 1] : Idx(0);
        const Idx up2 = sm.H[pos][hb + 2];
        if (rem < z1) {  // R
          pre2 += up2;
          --depth; --hb;
        } else {         // L
          rem -= z1;
          if (depth == 1) acc_from<K>(Mn + size_t(baseLL + pre2 + up2 + rem) * K, acc, mod);
          pre2 += up2 + sm.H[pos][hb + 1];
          ++depth; ++hb;
        }
      }
    }
  }
  // RR closures: every R at depth 1 of the high part (scanning up from p+1),
  // flipped to L, is a predecessor with pair RR (RV.hpp:70-82).  Its high base
  // is bm - S0 + S2 + H[q][h], S0/S2 the rank contributions of the positions
  // below q at their own and at +2 heights.
  {
    Idx S0 = 0, S2 = 0;
    int ha = h, depth = 1;
    const Idx offRR = sm.OFF[h + 2][PR_RR] + r;
    for (int q = p + 1; q <= W - 1 && depth > 0; ++q) {
      const uint32_t s = sym_at(hw, q);
      if (s == SYM_N) continue;  // N contributes nothing and keeps the height
      if (s == SYM_R) {
        const int hbq = ha + 1;
        if (depth == 1) acc_from<K>(Mn + size_t(bm - S0 + S2 + sm.H[q][h] + offRR) * K, acc, mod);
        S0 += sm.H[q][hbq];
        S2 += sm.H[q][hbq + 2];
        ha = hbq; ++depth;
      } else {
        const int hbq = ha - 1;
        S0 += sm.H[q][hbq] + (hbq > 0 ? sm.H[q][hbq - 1] : Idx(0));
        S2 += sm.H[q][hbq + 2] + sm.H[q][hbq + 1];
        ha = hbq; --depth;
      }
    }
  }
  if (p >= 2) {
    stk<K>(Bk + jK, acc);
  } else {
    // x holds NN + B; add the RR closures.
#pragma unroll
    for (int i = 0; i < K; ++i) x[i] = add_mod(x[i], acc[i], mod[i]);
    stk<K>(Mn + size_t(iNN) * K, x);
    if (a.blk_out_p1) {
#pragma unroll
      for (int i = 0; i < K; ++i) acc[i] = 0;
      stk<K>(Bk + jK, acc);
    }
  }
}

// ---- first row: initialiser and dot product ---------------------------------
// The state after the first row for one edge mask (GB.cu:1081-1096 semantics):
// cells p = W-1..1 only ever see pairs NN, RN, LN here because position p-1 is
// still untouched, so the included edge is NN->LR, RN->NR or LN->NL.
FDP_HD uint64_t first_row_state_dev(uint64_t mask, int W) {
  uint64_t m = uint64_t(SYM_R) << (2 * (W - 1));
  for (int p = W - 1; p >= 1; --p) {
    if (!((mask >> (p - 1)) & 1u)) continue;
    const int sh = 2 * (p - 1);
    const uint32_t pair = uint32_t(m >> sh) & 15u;
    const uint32_t np = pair == 0x0 ? 0x9u : (pair == 0x4 ? 0x1u : 0x2u);
    m = (m & ~(15ull << sh)) | (uint64_t(np) << sh);
  }
  return m;
}

template <typename Idx>
FDP_HD Idx rank_dev(uint64_t m, int W, const Idx (*H)[FDP_HT]) {
  Idx r = 0;
  int h = 1;
  for (int pos = W - 1; pos >= 0; --pos) {
    const uint32_t s = sym_at(m, pos);
    if (s > SYM_N) r += H[pos][h];
    if (s > SYM_R && h > 0) r += H[pos][h - 1];
    if (s == SYM_R) --h;
    else if (s == SYM_L) ++h;
  }
  return r;
}

}  // namespace fdp
