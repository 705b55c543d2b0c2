// Host-side tables, sizes and the byte model of the frontier DP.
#pragma once
#include <stdint.h>
#include <vector>

#include "fdp_core.cuh"

namespace fdp {

// H[w][h] in 64 bits for every width up to FDP_MAXW (GB.cu:172 build_full_dp):
// words of w symbols from height h to 0 whose heights stay in [0, cap].  The
// full space is cap = FDP_FULL_CAP; a smaller cap is the height-bounded space
// of the row-k prefix (the reference's build_bounded_dp, GB.cu:177-181).
#define FDP_FULL_CAP 1000
struct CountTable {
  uint64_t H[FDP_MAXW + 1][FDP_HT];
  int cap;
  explicit CountTable(int cap = FDP_FULL_CAP);
  uint64_t at(int w, int h) const { return (w < 0 || h < 0 || h >= FDP_HT || w > FDP_MAXW) ? 0 : H[w][h]; }
};
const CountTable &counts();                 // full space
const CountTable &counts_capped(int cap);   // cap in [1, FDP_HT-2]; full space above

uint64_t main_states(int W);     // H[W][1]
uint64_t blocked_states(int W);  // H[W-1][1]

// Index width needed for a frontier of width W: main ranks must fit the type.
bool needs_u64(int W);

// Fill the device table blob for width W in the space of height cap `cap`.
template <typename Idx>
void build_width_tables(int W, WidthTables<Idx> *out, int cap = FDP_FULL_CAP);

// Canonical rank / unrank (host reference of the device routines).
uint64_t rank_word(uint64_t word, int width, int cap = FDP_FULL_CAP);
uint64_t unrank_word(uint64_t rank, int width, int cap = FDP_FULL_CAP);
uint64_t main_states_capped(int W, int cap);     // H_cap[W][1]
uint64_t blocked_states_capped(int W, int cap);  // H_cap[W-1][1]

// The state reached by one first-row edge mask (GB.cu:1081-1096).
uint64_t first_row_state(uint64_t mask, int W);

// include_horizontal (TR.hpp:113-144): 0 invalid, 1 main, 2 blocked.
int include_horizontal(uint64_t m, int width, int p, uint64_t *out);

// Algorithmic bytes of one cell p for one modulus: the minimum traffic of the
// in-place sweep (the 4(M+D) + 4(Wm(p)+D) model without the blocked read at
// p = W-1, which is known zero, and without the blocked write at p = 1).
uint64_t cell_bytes(int W, int p, int cap = FDP_FULL_CAP);
// Algorithmic bytes of one row sweep p = W-1..1 in the space of height cap `cap`, one modulus.
uint64_t row_bytes(int W, int cap = FDP_FULL_CAP);
// Frontier transitions of one cell (main + blocked states), one modulus.
uint64_t cell_transitions(int W, int cap = FDP_FULL_CAP);

// Height caps of the bounded prefix: row r (r = 1, 2, ...) runs in the space
// of cap r + 1 while that space holds fewer than 95 % of the full space's
// states (the reference's bounded-height prefix, GB.cu:1825-1838).  Row 0 is
// the cap-1 space with every coefficient 1.
std::vector<int> bounded_prefix_caps(int W);

// Number of row sweeps a residue runs with the row-0 initialiser (prefixK = 1).
inline int sweep_rows(int W) { return W >= 3 ? W - 2 : 0; }

}  // namespace fdp
