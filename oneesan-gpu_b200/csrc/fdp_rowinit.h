// Row-k initialiser: the frontier-DP state after the first rows, computed
// directly instead of by row sweeps.
//
// The coefficient of a main word w after row r counts the edge sets of the
// strip of vertex rows 0..r (horizontal edges in those rows, vertical edges
// between them and down from row r) that form path pieces consistent with w:
// the start corner (row 0, position W-1) has degree 1, every other vertex 0 or
// 2, no cycles, and the pieces pair the down edges as w's parentheses do (read
// from position W-1 down, L opens, R closes, and the start corner's piece
// closes the initial height 1).  Reading w one position (grid column) at a time
// makes this a weighted finite automaton: its state is the cut between two
// columns, i.e. which of the r+1 horizontal edges cross it and what each one's
// piece must still do.  Each piece at the cut is one of:
//   O k : the piece of the k-th still-open arc of w (k = 0 is the start
//         corner's); it ends at an L already read (or at the start corner);
//   C   : two pieces that must meet further on: an open arc's piece and the
//         piece of the R that closed it;
//   U   : one piece with both ends at the cut.
// A state's number of O labels is the word's current height.  The weights are
// counts of column edge sets, so the automaton is the same for every modulus.
// This build derives the automaton itself, by enumerating the edge sets of one
// column; the reference ships generated tables for the same purpose (row-5 and
// row-6 automata, GB.cu:19-24, 874-1032).
#pragma once
#include <stdint.h>

#include <vector>

namespace fdp {

struct AutTrans {
  int from, to;  // interior state ids (from = -1: the initial state; to = -1: the final state)
  uint32_t weight;
};

struct RowAutomaton {
  int rows = 0;                 // vertex rows of the strip (r + 1)
  int nstates = 0;              // interior states
  std::vector<int> height;      // per state: number of open arcs
  std::vector<int> index;       // per state: index among the states of its height
  std::vector<int> per_height;  // states of each height 0..rows
  // Transitions by symbol (N, R, L): the first column (position W-1) from the
  // initial state, interior columns, and the last column (position 0) into the
  // final state.
  std::vector<AutTrans> first[3], inner[3], last[3];
};

// The automaton of the strip of `rows` vertex rows (1..7).
const RowAutomaton &row_automaton(int rows);

// Coefficient of main word w (width W >= 2) after row rows-1, modulo mod, by
// running the automaton over the word (host; used to check the tables).
uint32_t row_automaton_coeff(const RowAutomaton &a, uint64_t word, int W, uint32_t mod);

// How the state after row rows-1 is filled into a target space (width W,
// height cap `cap`): a word is its top P symbols (the prefix, positions
// W-1..S) and its bottom S = W - P symbols (the suffix).  In canonical order
// all completions of one prefix are contiguous, so with v_x the automaton
// vector after prefix x (over the states of x's end height h) and U_h the
// matrix of suffix vectors of every completion from h (in canonical order),
//   state[base_x + j] = (v_x . U_h)[j],
// one dense product per height.  Prefixes are built as a trie (level k from
// level k-1 by one column), suffix vectors level by level from the last
// column: the completions of k positions from height g are, in canonical
// order, N + (k-1 from g), R + (k-1 from g-1), L + (k-1 from g+1).
struct RowInitPlan {
  int W = 0, rows = 0, cap = 0, P = 0, S = 0, hmax = 0;
  uint64_t states = 0;  // main states of the target space
  std::vector<int> K;   // automaton states per height 0..rows
  // Prefix trie, levels 1..P: parent index in the previous level (-1 at level
  // 1), symbol, end height, and row among the level's prefixes of that height.
  std::vector<std::vector<int32_t>> parent, row;
  std::vector<std::vector<uint8_t>> sym, height;
  std::vector<std::vector<uint64_t>> rows_of;  // per level: prefixes per end height
  std::vector<uint64_t> base;                  // level P: first state of the prefix's block
  // C[k][g]: completions of k positions from height g in the target space
  std::vector<std::vector<uint64_t>> C;
  uint64_t mac = 0;  // multiply-adds of the products (per lane)
};

// Plan the fill for the strip of `rows` vertex rows into the target space
// (W, cap), choosing P to minimise the products' multiply-adds; prefixes whose
// heights leave 0..rows (zero vectors) are left out.
RowInitPlan plan_row_init(int W, int rows, int cap);

// Words of scratch per lane the device fill needs: two prefix levels and two
// suffix levels (the larger of each pair of consecutive levels).
uint64_t row_init_scratch_words(const RowInitPlan &plan);

// Device bytes of the fill's tables (automaton and prefix trie) for a plan;
// they stay resident once uploaded for that (W, rows, cap).
uint64_t row_init_table_bytes(const RowInitPlan &plan);

// The fill computed on the host for one modulus (reference for the device
// kernels and their tests): the whole target-space vector.
std::vector<uint32_t> row_init_fill_host(const RowInitPlan &plan, uint32_t mod);

}  // namespace fdp
