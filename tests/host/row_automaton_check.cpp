// Host check of the row-k initialiser (test infrastructure, built and run by
// tests/test_host_kernel_logic.py):
//   automaton : the column automaton's coefficient of every main word after
//               row r (r = 0..5) against the oracle's DP state after rows
//               1..r (forward recurrence from the row-0 initialiser);
//   fill      : the planned prefix x suffix fill (the computation the device
//               kernels perform) against the automaton, for every word of the
//               target spaces with caps rows, rows + 1 and the full space.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "fdp_host.h"
#include "fdp_rowinit.h"

extern "C" int oracle_forward_cell(int, int, uint32_t, const uint32_t *, const uint32_t *, uint32_t *, uint32_t *);
extern "C" uint64_t oracle_first_row_state(uint64_t, int);
extern "C" uint64_t oracle_rank(uint64_t, int);

using namespace fdp;

int main(int argc, char **argv) {
  const int wmax = argc > 1 ? atoi(argv[1]) : 10;
  const uint32_t mods[2] = {4294967291u, 2u};
  int bad = 0;
  uint64_t words = 0;
  for (int r = 0; r <= 5; ++r) {
    const RowAutomaton &A = row_automaton(r + 1);
    for (int W = 2; W <= wmax; ++W) {
      const uint32_t mod = mods[(r + W) % 2];
      const uint64_t M = main_states(W), D = blocked_states(W);
      std::vector<uint32_t> a(M, 0), b(D ? D : 1, 0), a2(M), b2(D ? D : 1);
      for (uint64_t mask = 0; mask < (1ull << (W - 1)); ++mask) a[oracle_rank(oracle_first_row_state(mask, W), W)] = 1 % mod;
      for (int row = 1; row <= r; ++row)
        for (int p = W - 1; p >= 1; --p) {
          oracle_forward_cell(W, p, mod, a.data(), b.data(), a2.data(), b2.data());
          a.swap(a2);
          b.swap(b2);
        }
      for (uint64_t i = 0; i < M; ++i, ++words)
        if (row_automaton_coeff(A, unrank_word(i, W), W, mod) != a[i]) {
          if (bad < 5) printf("automaton r=%d W=%d word %llu\n", r, W, (unsigned long long)i);
          ++bad;
        }
    }
  }
  printf("automaton words=%llu bad=%d\n", (unsigned long long)words, bad);
  for (int R = 1; R <= 6; ++R)
    for (int W = 2; W <= wmax + 1; ++W)
      for (int cap : {R, R + 1, FDP_FULL_CAP}) {
        const RowAutomaton &A = row_automaton(R);
        const uint32_t mod = mods[(R + W) % 2];
        const RowInitPlan pl = plan_row_init(W, R, cap);
        const std::vector<uint32_t> got = row_init_fill_host(pl, mod);
        for (uint64_t i = 0; i < pl.states; ++i)
          if (got[i] != row_automaton_coeff(A, unrank_word(i, W, cap), W, mod)) {
            if (bad < 10) printf("fill R=%d W=%d cap=%d P=%d word %llu\n", R, W, cap, pl.P, (unsigned long long)i);
            ++bad;
          }
      }
  printf("bad=%d\n", bad);
  return bad != 0;
}
