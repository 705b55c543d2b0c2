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
// Lane layout ("panels"): the K residues of a state (one per modulus) are
// split greedily into panels of 8, 4, 2 and 1 lanes; the panel with first lane
// L0 and width PW is its own array [N][PW] starting at word L0 * N, N = M or
// D.  A warp touching consecutive states of one panel reads one contiguous
// run of 32 * PW * 4 bytes, and one decoded index serves all K moduli.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fdp_core.cuh"

#define FDP_MAX_CAND 16  // closure predecessors of one blocked target: <= W/2 + 1 <= 15

namespace fdp {

// Closure predecessors of one c = N target at width W: LL sources are the
// depth-1 L's of the low word (p - 1 symbols), RR sources the depth-1 R's of
// the high part (W - 1 - p symbols); consecutive depth-1 symbols of one kind
// are separated by a symbol of the other kind, so there are at most
// ceil((p-1)/2) + ceil((W-1-p)/2) <= W/2 of them.  One slot of margin.
FDP_HD constexpr int cand_slots(int W) { return W / 2 + 1; }

struct CellArgs {
  const void *tables;  // WidthTables<Idx> in device memory
  uint32_t *main;      // K lanes of M states (panel layout)
  uint32_t *blk;       // K lanes of D states (panel layout)
  uint64_t items;      // D = blocked states
  uint64_t mstates;    // M = main states
  uint32_t mod[16];
  int W, p;
  int blk_in_zero;     // blocked input known to be zero (first cell of a row sweep)
  int blk_out_p1;      // at p = 1 store the (all-zero) blocked output
  int cap;             // height cap of the state space (FDP_FULL_CAP: unbounded)
  int lane_items;      // items per lane of one warp chunk (the chunk is 32 * lane_items indices)
  int share_prefix;    // decode the prefix a warp chunk shares once per chunk
  int compact;         // small-p cells: 1 = a chunk's items updated grouped by centre type
                       // (lane_items <= FDP_REC_MAX_ITEMS), 2 = grouped with carry-over queues
};

struct FirstRowArgs {
  const void *tables;
  uint32_t *main;                 // K lanes of M states (panel layout)
  unsigned long long *acc;        // [K] 64-bit accumulators (dot product)
  uint64_t mstates;
  uint32_t mod[16];
  int W;
};

// ---- panel layout -----------------------------------------------------------
// Panel widths: greedy 8, 4, 2, 1 (8-wide panels measured fastest on B200).
template <int K, int L0>
struct PanelW {
  static constexpr int value = (K - L0 >= 8) ? 8 : (K - L0 >= 4) ? 4 : ((K - L0 >= 2) ? 2 : 1);
};

// Bytes a panel array's base must be aligned to: one word of the widest panel
// (an 8-lane word is one 32-byte access).  Panels start at word L0 * N with L0
// a multiple of their width, so the base alignment carries to every panel.
FDP_HD constexpr int panel_align_bytes(int K) { return K >= 8 ? 32 : (K >= 4 ? 16 : (K >= 2 ? 8 : 4)); }
inline bool panel_aligned(int K, const void *base) {
  return (reinterpret_cast<uintptr_t>(base) & uintptr_t(panel_align_bytes(K) - 1)) == 0;
}

// One state word of a panel.  On the device an 8-lane word is a single 256-bit
// access (ld/st.global.v8.b32, sm_100): half the load and store instructions
// of two 128-bit halves, and one L1 request per 32-byte sector (measured at
// n = 22, 14 lanes: pass 16.73 -> 16.48 s, the small-p cells 2-5 % faster).
template <int PW>
FDP_HD void ld_panel(const uint32_t *p, uint32_t *x) {
#if defined(__CUDA_ARCH__)
  if constexpr (PW == 8) {
    asm volatile("ld.global.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(x[0]), "=r"(x[1]), "=r"(x[2]), "=r"(x[3]), "=r"(x[4]), "=r"(x[5]), "=r"(x[6]), "=r"(x[7])
                 : "l"(p));
    return;
  }
#endif
  if constexpr (PW == 8) {
    const uint4 t = reinterpret_cast<const uint4 *>(p)[0];
    const uint4 u = reinterpret_cast<const uint4 *>(p)[1];
    x[0] = t.x; x[1] = t.y; x[2] = t.z; x[3] = t.w;
    x[4] = u.x; x[5] = u.y; x[6] = u.z; x[7] = u.w;
  } else if constexpr (PW == 4) {
    const uint4 t = *reinterpret_cast<const uint4 *>(p);
    x[0] = t.x; x[1] = t.y; x[2] = t.z; x[3] = t.w;
  } else if constexpr (PW == 2) {
    const uint2 t = *reinterpret_cast<const uint2 *>(p);
    x[0] = t.x; x[1] = t.y;
  } else {
    x[0] = *p;
  }
}

template <int PW>
FDP_HD void st_panel(uint32_t *p, const uint32_t *x) {
#if defined(__CUDA_ARCH__)
  if constexpr (PW == 8) {
    asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"(x[0]), "r"(x[1]),
                 "r"(x[2]), "r"(x[3]), "r"(x[4]), "r"(x[5]), "r"(x[6]), "r"(x[7])
                 : "memory");
    return;
  }
#endif
  if constexpr (PW == 8) {
    reinterpret_cast<uint4 *>(p)[0] = make_uint4(x[0], x[1], x[2], x[3]);
    reinterpret_cast<uint4 *>(p)[1] = make_uint4(x[4], x[5], x[6], x[7]);
  } else if constexpr (PW == 4) *reinterpret_cast<uint4 *>(p) = make_uint4(x[0], x[1], x[2], x[3]);
  else if constexpr (PW == 2) *reinterpret_cast<uint2 *>(p) = make_uint2(x[0], x[1]);
  else *p = x[0];
}

// Word address of lane L0's panel for state s.
template <int K, int L0>
FDP_HD size_t panel_word(size_t N, size_t s) {
  return size_t(L0) * N + s * size_t(PanelW<K, L0>::value);
}

// All K lanes of state s (used by the first-row kernels).
template <int K, int L0 = 0>
FDP_HD void ld_lanes(const uint32_t *base, size_t N, size_t s, uint32_t *x) {
  if constexpr (L0 < K) {
    constexpr int PW = PanelW<K, L0>::value;
    ld_panel<PW>(base + panel_word<K, L0>(N, s), x + L0);
    ld_lanes<K, L0 + PW>(base, N, s, x);
  }
}

template <int K, int L0 = 0>
FDP_HD void st_lanes(uint32_t *base, size_t N, size_t s, const uint32_t *x) {
  if constexpr (L0 < K) {
    constexpr int PW = PanelW<K, L0>::value;
    st_panel<PW>(base + panel_word<K, L0>(N, s), x + L0);
    st_lanes<K, L0 + PW>(base, N, s, x);
  }
}

// Spans: runs of consecutive panels holding at most 8 lanes together (K = 14:
// {0-7}, {8-13}).  The cell kernel reads and writes a state one span at a
// time and issues all loads of a span before it uses any of them, so a lane
// count of several small panels costs no more dependent load phases than one
// of 8-wide panels.
FDP_HD constexpr int span_end_of(int K, int L0) {
  int l = L0, w = 0;
  while (l < K) {
    const int pw = (K - l >= 8) ? 8 : (K - l >= 4) ? 4 : ((K - l >= 2) ? 2 : 1);
    if (w + pw > 8) break;
    w += pw;
    l += pw;
  }
  return l;
}

template <int K>
FDP_HD constexpr int span_count() {
  int n = 0;
  for (int l = 0; l < K; l = span_end_of(K, l)) ++n;
  return n;
}

// Lanes [L0, LE) of state s (LE a span end) into x[0 .. LE-L0).
template <int K, int L0, int LE, int X0 = L0>
FDP_HD void ld_span(const uint32_t *base, size_t N, size_t s, uint32_t *x) {
  if constexpr (L0 < LE) {
    constexpr int PW = PanelW<K, L0>::value;
    ld_panel<PW>(base + panel_word<K, L0>(N, s), x + (L0 - X0));
    ld_span<K, L0 + PW, LE, X0>(base, N, s, x);
  }
}

template <int K, int L0, int LE, int X0 = L0>
FDP_HD void st_span(uint32_t *base, size_t N, size_t s, const uint32_t *x) {
  if constexpr (L0 < LE) {
    constexpr int PW = PanelW<K, L0>::value;
    st_panel<PW>(base + panel_word<K, L0>(N, s), x + (L0 - X0));
    st_span<K, L0 + PW, LE, X0>(base, N, s, x);
  }
}

// ---- shared-memory copies of the width tables ------------------------------
// Heights are trimmed to FDP_HS: a legal word of at most 28 symbols never
// rises above 14, and the kernel looks at most 2 heights above a legal one.
#define FDP_HS 18
template <typename Idx>
struct CellSmem {
  StepT<Idx> S[FDP_MAXW][FDP_HS];
  Idx H[FDP_MAXW + 1][FDP_HS];
  Idx OFF[FDP_HS][PR_COUNT];
};

// The decoded head of a work item: blocked index j, its high prefix (main base
// bm, end height h, high symbols hw with main position q at bits 2*(q-p-1)),
// the centre symbol c at blocked position p-1 (0 = N, 1 = R, 2 = L) and the
// low rank r.
template <typename Idx>
struct Head {
  Idx j, r, bm;
  uint64_t hw;
  int h, c;
};

// A c = N item after its closure sources were staged in the candidate slots.
template <typename Idx>
struct NItem {
  Idx j;
  Idx iNN, iLR, iRL;  // owned NN and LR words, RL source
  int hasRL;          // the RL source exists (h > 0, p >= 2)
  int hasLR;          // the LR target exists (always, except at the height cap)
  int nc;             // closure sources in the candidate slots
};

// A partly decoded blocked prefix: positions above `pos` are decoded (main
// base bm, height h, high symbols hw), and j - sub is the rank left for
// blocked positions pos..0.
template <typename Idx>
struct Prefix {
  Idx sub, bm;
  uint64_t hw;
  int pos, h;
};

template <typename Idx>
FDP_HD Prefix<Idx> empty_prefix(const CellArgs &a) {
  return Prefix<Idx>{Idx(0), Idx(0), 0ull, a.W - 2, 1};
}

// The prefix shared by every blocked index in [jb, jl].  Ranks are
// lexicographic from the top position down, so every word ranked between two
// words carries the top symbols those two have in common: one walk of jb and
// jl in step, stopping where they part, decodes that part for the whole range.
template <typename Idx>
FDP_HD Prefix<Idx> shared_prefix(const CellArgs &a, const CellSmem<Idx> &sm, const Idx jb, const Idx jl) {
  Idx r0 = jb, r1 = jl, bm = 0;
  int h = 1, pos = a.W - 2;
  uint64_t hw = 0;
  for (; pos >= a.p; --pos) {
    const StepT<Idx> s = sm.S[pos][h];
    const uint32_t s0 = r0 >= s.t2 ? SYM_L : (r0 >= s.t1 ? SYM_R : SYM_N);
    const uint32_t s1 = r1 >= s.t2 ? SYM_L : (r1 >= s.t1 ? SYM_R : SYM_N);
    if (s0 != s1) break;
    const Idx t = s0 == SYM_L ? s.t2 : (s0 == SYM_R ? s.t1 : Idx(0));
    r0 -= t;
    r1 -= t;
    bm += s0 == SYM_L ? s.cL : (s0 == SYM_R ? s.cR : Idx(0));
    h += s0 == SYM_L ? 1 : (s0 == SYM_R ? -1 : 0);
    hw = (hw << 2) | s0;
  }
  return Prefix<Idx>{Idx(jb - r0), bm, hw, pos, h};
}

// Decode blocked index j at cell p, starting from a prefix pf that j shares:
// the rest of the high prefix (blocked positions pf.pos..p, top-down), then
// the centre symbol and the low rank.
template <typename Idx>
FDP_HD Head<Idx> decode_head(const CellArgs &a, const CellSmem<Idx> &sm, const Idx j, const Prefix<Idx> &pf) {
  const int p = a.p;
  Idx r = j - pf.sub, bm = pf.bm;
  int h = pf.h;
  uint64_t hw = pf.hw;
  for (int pos = pf.pos; pos >= p; --pos) {
    const StepT<Idx> s = sm.S[pos][h];
    const bool ge1 = r >= s.t1, ge2 = r >= s.t2;
    r -= ge2 ? s.t2 : (ge1 ? s.t1 : Idx(0));
    bm += ge2 ? s.cL : (ge1 ? s.cR : Idx(0));
    h += ge2 ? 1 : (ge1 ? -1 : 0);
    hw = (hw << 2) | uint64_t(ge2 ? SYM_L : (ge1 ? SYM_R : SYM_N));
  }
  int c = 0;
  const Idx bN = sm.H[p - 1][h];
  if (r >= bN) {
    r -= bN;
    const Idx bR = h > 0 ? sm.H[p - 1][h - 1] : Idx(0);
    if (r < bR) c = 1;
    else { r -= bR; c = 2; }
  }
  return Head<Idx>{j, r, bm, hw, h, c};
}

// Every closure predecessor (its main index) of a c = N head, handed to
// on_cand: LL sources scanning the low word down, then RR sources scanning the
// high part up.
template <typename Idx, typename OnCand>
FDP_HD void for_each_closure(const CellArgs &a, const CellSmem<Idx> &sm, const Head<Idx> &hd, OnCand &&on_cand) {
  const int p = a.p, h = hd.h;
  const Idx r = hd.r, bm = hd.bm;
  // LL closures (p >= 3): every L at depth 1 of the low word, flipped to R,
  // is a predecessor with pair LL (RV.hpp:49-69 enumerates the same set).
  // Its rank from height h+2 is the +2-shifted prefix rank, plus H[pos][hb+2]
  // for the R, plus the unchanged remainder below.
  if (p >= 3) {
    const Idx baseLL = bm + sm.OFF[h][PR_LL];
    Idx rem = r, pre2 = 0;
    int hb = h, depth = 1, mx = h;  // mx: highest height so far (the predecessor sits 2 higher)
    for (int pos = p - 2; pos >= 0 && depth > 0; --pos) {
      const Idx z0 = sm.H[pos][hb];
      if (rem < z0) continue;  // N: no contribution at either height
      rem -= z0;
      const Idx z1 = hb > 0 ? sm.H[pos][hb - 1] : Idx(0);
      const Idx up2 = sm.H[pos][hb + 2];
      if (rem < z1) {  // R
        pre2 += up2;
        --depth; --hb;
      } else {         // L
        rem -= z1;
        if (depth == 1 && mx + 2 <= a.cap) on_cand(baseLL + pre2 + up2 + rem);
        pre2 += up2 + sm.H[pos][hb + 1];
        ++depth; ++hb;
        mx = hb > mx ? hb : mx;
      }
    }
  }
  // RR closures: every R at depth 1 of the high part (scanning up from p+1),
  // flipped to L, is a predecessor with pair RR (RV.hpp:70-82).  Its high base
  // is bm - S0 + S2 + H[q][h], S0/S2 the rank contributions of the positions
  // below q at their own and at +2 heights.  N symbols are skipped with the
  // non-N bit mask.
  const Idx offRR = sm.OFF[h + 2][PR_RR] + r;
  const uint64_t hw = hd.hw;
  uint64_t nn = (hw | (hw >> 1)) & 0x5555555555555555ull;
  Idx S0 = 0, S2 = 0;
  int ha = h, depth = 1, mx = h;  // mx: highest height below q (the predecessor sits 2 higher)
  while (nn && depth > 0) {
#if defined(__CUDA_ARCH__)
    const int b = __ffsll((long long)nn) - 1;
#else
    const int b = __builtin_ctzll(nn);
#endif
    nn &= nn - 1;
    const int q = p + 1 + (b >> 1);
    if (((hw >> b) & 3u) == SYM_R) {
      const int hbq = ha + 1;
      if (depth == 1 && mx + 2 <= a.cap) on_cand(bm - S0 + S2 + sm.H[q][h] + offRR);
      S0 += sm.H[q][hbq];
      S2 += sm.H[q][hbq + 2];
      ha = hbq; ++depth;
      mx = hbq > mx ? hbq : mx;
    } else {
      const int hbq = ha - 1;
      S0 += sm.H[q][hbq] + (hbq > 0 ? sm.H[q][hbq - 1] : Idx(0));
      S2 += sm.H[q][hbq + 2] + sm.H[q][hbq + 1];
      ha = hbq; --depth;
    }
  }
}

// c = R / L, one span at a time (X = NR/NL, Y = RN/LN):
//   p >= 2:  X' = X + Y + B, B' = X
//   p == 1:  (c = R only) NR' = NR + RN + B, RN' = RN + NR, B' = 0 if stored
template <typename Idx, int K, int L0 = 0>
FDP_HD void apply_x(const CellArgs &a, const Idx iA, const Idx iB, const Idx j) {
  if constexpr (L0 < K) {
    constexpr int LE = span_end_of(K, L0), G = LE - L0;
    uint32_t *const Mn = a.main;
    uint32_t *const Bk = a.blk;
    const size_t M = a.mstates, D = a.items;
    const uint32_t *mod = a.mod + L0;
    uint32_t x[G], y[G], z[G];
    ld_span<K, L0, LE>(Mn, M, size_t(iA), x);
    ld_span<K, L0, LE>(Mn, M, size_t(iB), y);
    if (!a.blk_in_zero) {
      uint32_t b[G];
      ld_span<K, L0, LE>(Bk, D, size_t(j), b);
#pragma unroll
      for (int i = 0; i < G; ++i) z[i] = add_mod(add_mod(x[i], y[i], mod[i]), b[i], mod[i]);
    } else {
#pragma unroll
      for (int i = 0; i < G; ++i) z[i] = add_mod(x[i], y[i], mod[i]);
    }
    st_span<K, L0, LE>(Mn, M, size_t(iA), z);
    if (a.p >= 2) {
      st_span<K, L0, LE>(Bk, D, size_t(j), x);
    } else {
#pragma unroll
      for (int i = 0; i < G; ++i) z[i] = add_mod(y[i], x[i], mod[i]);
      st_span<K, L0, LE>(Mn, M, size_t(iB), z);
      if (a.blk_out_p1) {
#pragma unroll
        for (int i = 0; i < G; ++i) z[i] = 0;
        st_span<K, L0, LE>(Bk, D, size_t(j), z);
      }
    }
    apply_x<Idx, K, LE>(a, iA, iB, j);
  }
}

// The two main words of a c = R/L head: the owned NR/NL word and the RN/LN
// source (item_x's operands).
template <typename Idx>
FDP_HD void x_words(const CellSmem<Idx> &sm, const Head<Idx> &hd, Idx &ia, Idx &ib) {
  const Idx *off = sm.OFF[hd.h];
  ia = hd.bm + off[hd.c == 1 ? PR_NR : PR_NL] + hd.r;
  ib = hd.bm + off[hd.c == 1 ? PR_RN : PR_LN] + hd.r;
}

template <typename Idx, int K>
FDP_HD void item_x(const CellArgs &a, const CellSmem<Idx> &sm, const Head<Idx> &hd) {
  Idx ia, ib;
  x_words<Idx>(sm, hd, ia, ib);
  apply_x<Idx, K>(a, ia, ib, hd.j);
}

// c = N with the closure sources staged in cand[i * cstride], one span at a
// time:
//   p >= 2:  NN' = NN + B, LR' = LR + NN, B' = RL + closures
//   p == 1:  NN' = NN + B + RR closures, LR' = LR + NN, B' = 0 if stored
// The three streamed words NN, LR and B are loaded before the first store: a
// load placed after a store cannot be moved above it (the compiler must
// assume they may alias), so this order costs one memory round trip where
// load / store / load costs two.  RL and the closure sources follow, two at a
// time.  None of those words is written by another item of the cell.
template <typename Idx, int K, int L0 = 0>
FDP_HD void apply_n(const CellArgs &a, const NItem<Idx> &it, const Idx *cand, int cstride) {
  if constexpr (L0 < K) {
    constexpr int LE = span_end_of(K, L0), G = LE - L0;
    uint32_t *const Mn = a.main;
    uint32_t *const Bk = a.blk;
    const size_t M = a.mstates, D = a.items;
    const uint32_t *mod = a.mod + L0;
    const size_t jj = size_t(it.j);
    uint32_t x[G], acc[G];
    {
      uint32_t y[G], b[G];
      ld_span<K, L0, LE>(Mn, M, size_t(it.iNN), x);
      if (!a.blk_in_zero) ld_span<K, L0, LE>(Bk, D, jj, b);
      else {
#pragma unroll
        for (int i = 0; i < G; ++i) b[i] = 0;
      }
      if (it.hasLR) ld_span<K, L0, LE>(Mn, M, size_t(it.iLR), y);
      if (it.hasLR) {
#pragma unroll
        for (int i = 0; i < G; ++i) y[i] = add_mod(y[i], x[i], mod[i]);
        st_span<K, L0, LE>(Mn, M, size_t(it.iLR), y);
      }
#pragma unroll
      for (int i = 0; i < G; ++i) x[i] = add_mod(x[i], b[i], mod[i]);
    }
#pragma unroll
    for (int i = 0; i < G; ++i) acc[i] = 0;
    if (a.p >= 2) {
      st_span<K, L0, LE>(Mn, M, size_t(it.iNN), x);
      if (it.hasRL) ld_span<K, L0, LE>(Mn, M, size_t(it.iRL), acc);
    }
    int k = 0;
    for (; k + 1 < it.nc; k += 2) {
      uint32_t u[G], v[G];
      ld_span<K, L0, LE>(Mn, M, size_t(cand[k * cstride]), u);
      ld_span<K, L0, LE>(Mn, M, size_t(cand[(k + 1) * cstride]), v);
#pragma unroll
      for (int i = 0; i < G; ++i) acc[i] = add_mod(add_mod(acc[i], u[i], mod[i]), v[i], mod[i]);
    }
    if (k < it.nc) {
      uint32_t u[G];
      ld_span<K, L0, LE>(Mn, M, size_t(cand[k * cstride]), u);
#pragma unroll
      for (int i = 0; i < G; ++i) acc[i] = add_mod(acc[i], u[i], mod[i]);
    }
    if (a.p >= 2) {
      st_span<K, L0, LE>(Bk, D, jj, acc);
    } else {
#pragma unroll
      for (int i = 0; i < G; ++i) x[i] = add_mod(x[i], acc[i], mod[i]);
      st_span<K, L0, LE>(Mn, M, size_t(it.iNN), x);
      if (a.blk_out_p1) {
#pragma unroll
        for (int i = 0; i < G; ++i) acc[i] = 0;
        st_span<K, L0, LE>(Bk, D, jj, acc);
      }
    }
    apply_n<Idx, K, LE>(a, it, cand, cstride);
  }
}

// Whether the cell kernel for K lanes stages closure candidates in shared
// memory (several spans) or sums them while scanning (one span).
template <int K>
FDP_HD constexpr bool stages_candidates() { return span_count<K>() > 1; }

// c = N, one span (K <= 8): same formulas and load order as apply_n; the
// closure sources are added as the scans find them.
template <typename Idx, int K>
FDP_HD void item_n_one_span(const CellArgs &a, const CellSmem<Idx> &sm, const Head<Idx> &hd) {
  const int p = a.p;
  uint32_t *const Mn = a.main;
  uint32_t *const Bk = a.blk;
  const size_t M = a.mstates, D = a.items;
  const uint32_t *mod = a.mod;
  const Idx *off = sm.OFF[hd.h];
  const Idx iNN = hd.bm + off[PR_NN] + hd.r;
  uint32_t x[K], acc[K];
  {
    const Idx iLR = hd.bm + off[PR_LR] + hd.r;
    const bool lr = hd.h + 1 <= a.cap;  // the LR target exists below the height cap
    uint32_t y[K], b[K];
    ld_span<K, 0, K>(Mn, M, size_t(iNN), x);
    if (!a.blk_in_zero) ld_span<K, 0, K>(Bk, D, size_t(hd.j), b);
    else {
#pragma unroll
      for (int i = 0; i < K; ++i) b[i] = 0;
    }
    if (lr) ld_span<K, 0, K>(Mn, M, size_t(iLR), y);
    if (lr) {
#pragma unroll
      for (int i = 0; i < K; ++i) y[i] = add_mod(y[i], x[i], mod[i]);
      st_span<K, 0, K>(Mn, M, size_t(iLR), y);
    }
#pragma unroll
    for (int i = 0; i < K; ++i) x[i] = add_mod(x[i], b[i], mod[i]);
  }
#pragma unroll
  for (int i = 0; i < K; ++i) acc[i] = 0;
  if (p >= 2) {
    st_span<K, 0, K>(Mn, M, size_t(iNN), x);
    if (hd.h > 0) ld_span<K, 0, K>(Mn, M, size_t(hd.bm + off[PR_RL] + hd.r), acc);
  }
  for_each_closure<Idx>(a, sm, hd, [&](Idx idx) {
    uint32_t u[K];
    ld_span<K, 0, K>(Mn, M, size_t(idx), u);
#pragma unroll
    for (int i = 0; i < K; ++i) acc[i] = add_mod(acc[i], u[i], mod[i]);
  });
  if (p >= 2) {
    st_span<K, 0, K>(Bk, D, size_t(hd.j), acc);
  } else {
#pragma unroll
    for (int i = 0; i < K; ++i) x[i] = add_mod(x[i], acc[i], mod[i]);
    st_span<K, 0, K>(Mn, M, size_t(iNN), x);
    if (a.blk_out_p1) {
#pragma unroll
      for (int i = 0; i < K; ++i) acc[i] = 0;
      st_span<K, 0, K>(Bk, D, size_t(hd.j), acc);
    }
  }
}

template <typename Idx, int K>
FDP_HD void item_n(const CellArgs &a, const CellSmem<Idx> &sm, const Head<Idx> &hd, Idx *cand, int cstride) {
  if constexpr (!stages_candidates<K>()) {
    (void)cand; (void)cstride;
    item_n_one_span<Idx, K>(a, sm, hd);
  } else {
    const Idx *off = sm.OFF[hd.h];
    NItem<Idx> it;
    it.j = hd.j;
    it.iNN = hd.bm + off[PR_NN] + hd.r;
    it.iLR = hd.bm + off[PR_LR] + hd.r;
    it.iRL = hd.bm + off[PR_RL] + hd.r;
    it.hasRL = (hd.h > 0 && a.p >= 2) ? 1 : 0;
    it.hasLR = (hd.h + 1 <= a.cap) ? 1 : 0;
    int n = 0;
    for_each_closure<Idx>(a, sm, hd, [&](Idx idx) { cand[(n++) * cstride] = idx; });
    it.nc = n;
    apply_n<Idx, K>(a, it, cand, cstride);
  }
}

// Decoded heads of one warp chunk in shared memory (structure of arrays of
// `cap` entries): the compacted kernel path stores every head of a chunk
// first, then updates the c = R/L items and the c = N items each with whole
// warps.
#define FDP_REC_MAX_ITEMS 4  // states per lane of a compacted chunk, at most
template <typename Idx>
FDP_HD constexpr size_t head_rec_entry_bytes() {
  return sizeof(uint64_t) + 3 * sizeof(Idx) + sizeof(uint32_t);
}

template <typename Idx>
struct HeadRecs {
  unsigned char *base;  // hw[cap] (u64), then j[cap], r[cap], bm[cap] (Idx), then hc[cap] = h | c << 8
  int cap;
  FDP_HD uint64_t *hw() const { return reinterpret_cast<uint64_t *>(base); }
  FDP_HD Idx *idx(int field) const { return reinterpret_cast<Idx *>(base + size_t(cap) * 8) + field * cap; }
  FDP_HD uint32_t *hc() const { return reinterpret_cast<uint32_t *>(base + size_t(cap) * (8 + 3 * sizeof(Idx))); }
  FDP_HD void put(int k, const Head<Idx> &h) const {
    hw()[k] = h.hw;
    idx(0)[k] = h.j;
    idx(1)[k] = h.r;
    idx(2)[k] = h.bm;
    hc()[k] = uint32_t(h.h) | (uint32_t(h.c) << 8);
  }
  FDP_HD Head<Idx> get(int k) const {
    const uint32_t v = hc()[k];
    return Head<Idx>{idx(0)[k], idx(1)[k], idx(2)[k], hw()[k], int(v & 255u), int(v >> 8)};
  }
};

// Carry-over stores of the grouped small-p path, one per warp.  Heads decoded
// from successive chunks queue by centre type until 32 of one type wait, so
// every grouped update runs on a full warp (grouping per chunk alone leaves a
// third of the lanes idle at p <= 6).  Each queue is a stack of at most 63
// entries (31 carried over + 32 new): c = R/L items as their three word
// indices, c = N items as heads with the end height packed above the high
// symbols (at most 2 x 26 bits for W <= 28, p >= 1).
#define FDP_CARRY_CAP 64
template <typename Idx>
FDP_HD constexpr size_t carry_rec_bytes() {
  return size_t(FDP_CARRY_CAP) * (sizeof(uint64_t) + 6 * sizeof(Idx));
}

template <typename Idx>
struct CarryRecs {
  unsigned char *base;  // hwh[64] (u64), then x: a[64], b[64], j[64]; n: j[64], r[64], bm[64] (Idx)
  FDP_HD uint64_t *hwh() const { return reinterpret_cast<uint64_t *>(base); }
  FDP_HD Idx *f(int field) const {
    return reinterpret_cast<Idx *>(base + size_t(FDP_CARRY_CAP) * 8) + field * FDP_CARRY_CAP;
  }
  FDP_HD void put_x(int k, Idx ia, Idx ib, Idx j) const {
    f(0)[k] = ia;
    f(1)[k] = ib;
    f(2)[k] = j;
  }
  FDP_HD void put_n(int k, const Head<Idx> &h) const {
    hwh()[k] = h.hw | (uint64_t(h.h) << 56);
    f(3)[k] = h.j;
    f(4)[k] = h.r;
    f(5)[k] = h.bm;
  }
  FDP_HD Head<Idx> get_n(int k) const {
    const uint64_t v = hwh()[k];
    return Head<Idx>{f(3)[k], f(4)[k], f(5)[k], v & ((1ull << 56) - 1ull), int(v >> 56), 0};
  }
};

// One work item: decode blocked index j (which shares prefix pf) and update
// the words it owns.
template <typename Idx, int K>
FDP_HD void cell_item(const CellArgs &a, const CellSmem<Idx> &sm, const Idx j, const Prefix<Idx> &pf, Idx *cand,
                      int cstride) {
  const Head<Idx> hd = decode_head<Idx>(a, sm, j, pf);
  if (hd.c != 0) item_x<Idx, K>(a, sm, hd);
  else item_n<Idx, K>(a, sm, hd, cand, cstride);
}

// ---- first row ----------------------------------------------------------------
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
