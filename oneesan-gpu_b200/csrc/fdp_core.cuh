// Frontier-DP state algebra and canonical-rank index arithmetic, shared by the
// sm_100a kernels and the host planner.
//
// State model (restated from src/common/gridfp_transition.hpp:20-146 of the
// reference):
//   * A main state is a word of W = n+1 two-bit symbols N=0, R=1, L=2 at
//     positions W-1 (top) .. 0 (bottom).  Reading top-down, L raises the height
//     by one and R lowers it; the height starts at 1 and ends at 0.
//   * A blocked state is the same with W-1 symbols.  It only lives between two
//     consecutive cells of a row sweep.
//   * Coefficients are uint32 residues; arrays are in canonical lexicographic
//     rank order (N<R<L), the order of GB.cu:1568 rank_full.
//
// Block structure used by the pull kernel (this file's own derivation): for a
// cell p, split a main word into  high = positions W-1..p+1 (ending at height
// h), pair = (p, p-1) and low = positions p-2..0.  In canonical order all
// completions of one high prefix are contiguous and, within that run, the nine
// pair sub-blocks are contiguous ranges of low words; the sub-block for pair
// (a,b) holds every low word of length p-1 starting at height h+d(a)+d(b).  A
// blocked word at the same cell splits into the same high prefix (blocked
// positions W-2..p), one centre symbol c at p-1 and the same low part.  Hence
// every non-closure move of the per-cell operator is "sub-block += sub-block
// at the same low rank", and the two closures (LL, RR) change one low or one
// high symbol, which this header turns into closed-form rank offsets.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define FDP_HD __host__ __device__ __forceinline__
#else
#define FDP_HD inline
#endif

#define FDP_MAXW 28   // widest frontier handled (n <= 27), as the reference (GB.cu:28)
#define FDP_HT 34     // height dimension of the count tables (heights 0..33)

namespace fdp {

enum : uint32_t { SYM_N = 0, SYM_R = 1, SYM_L = 2 };

// Lexicographic order of the nine legal symbol pairs (a at p, b at p-1).
enum : int { PR_NN = 0, PR_NR, PR_NL, PR_RN, PR_RR, PR_RL, PR_LN, PR_LR, PR_LL, PR_COUNT };

// One step of unranking a blocked prefix at blocked position `pos` and height h:
//   rank < t1            -> symbol N
//   t1 <= rank < t2      -> symbol R  (rank -= t1, main base += cR, h--)
//   t2 <= rank           -> symbol L  (rank -= t2, main base += cL, h++)
// cR/cL are the main-rank contributions of the same symbol at main position
// pos+1, so the main-rank base of the high prefix falls out of the same walk.
template <typename Idx>
struct StepT {
  Idx t1, t2, cR, cL;
};

// Device-resident per-width tables (one blob per frontier width W).
template <typename Idx>
struct WidthTables {
  Idx H[FDP_MAXW + 1][FDP_HT];                // H[w][h]: words of w symbols from height h to 0
  StepT<Idx> S[FDP_MAXW][FDP_HT];             // blocked-prefix unrank steps
  Idx OFF[FDP_MAXW][FDP_HT][PR_COUNT];        // OFF[p][h][pair]: sub-block offset in a high run
};

FDP_HD uint32_t sym_at(uint64_t w, int pos) { return uint32_t(w >> (2 * pos)) & 3u; }

// d(a)+d(b) for the pair index, and the intermediate height check.
FDP_HD int pair_first(int pr) { return pr / 3; }
FDP_HD int pair_second(int pr) { return pr % 3; }
FDP_HD int sym_delta(int s) { return s == (int)SYM_N ? 0 : (s == (int)SYM_R ? -1 : 1); }

// Addition modulo p for a, b in [0, p), p in [2, 2^32): exact for every modulus
// (GB.cu:1181 uses the same conditional-subtract identity).
FDP_HD uint32_t add_mod(uint32_t a, uint32_t b, uint32_t p) {
  uint32_t s = a + b;
  return (s < a || s >= p) ? s - p : s;
}

// One step of a walk that unranks a main word in one state space (count table
// F) and ranks it in another (count table T) at the same time: the symbol at
// `pos` follows from the residual rank r at height h (N below F[pos][h], then
// R, then L), and its rank contribution in T is added to j.  Used to move a
// state vector between height-bounded spaces.
template <typename T>
FDP_HD void expand_step(const T (*F)[FDP_HT], const T (*Tt)[FDP_HT], int pos, uint64_t &r, uint64_t &j, int &h) {
  const uint64_t zN = F[pos][h];
  if (r < zN) return;  // N: no contribution in either space
  r -= zN;
  const uint64_t zR = h > 0 ? uint64_t(F[pos][h - 1]) : 0ull;
  if (r < zR) {  // R
    j += Tt[pos][h];
    --h;
    return;
  }
  r -= zR;  // L
  j += uint64_t(Tt[pos][h]) + (h > 0 ? uint64_t(Tt[pos][h - 1]) : 0ull);
  ++h;
}

}  // namespace fdp
