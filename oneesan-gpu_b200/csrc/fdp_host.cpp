// Host-side count tables, canonical rank, device table blobs and the byte model.
#include "fdp_host.h"

#include <string.h>

#include <vector>

namespace fdp {

CountTable::CountTable(int c) : cap(c) {
  memset(H, 0, sizeof(H));
  H[0][0] = 1;
  for (int w = 1; w <= FDP_MAXW; ++w)
    for (int h = 0; h < FDP_HT && h <= cap; ++h) {
      uint64_t x = H[w - 1][h];
      if (h > 0) x += H[w - 1][h - 1];
      if (h + 1 < FDP_HT && h + 1 <= cap) x += H[w - 1][h + 1];
      H[w][h] = x;
    }
}

const CountTable &counts() {
  static const CountTable t(FDP_FULL_CAP);
  return t;
}

const CountTable &counts_capped(int cap) {
  static const std::vector<CountTable> tabs = [] {
    std::vector<CountTable> v;
    for (int c = 0; c < FDP_HT; ++c) v.emplace_back(c);
    return v;
  }();
  if (cap < 1 || cap >= FDP_HT - 1) return counts();
  return tabs[size_t(cap)];
}

uint64_t main_states_capped(int W, int cap) { return counts_capped(cap).at(W, 1); }
uint64_t blocked_states_capped(int W, int cap) { return counts_capped(cap).at(W - 1, 1); }

uint64_t main_states(int W) { return counts().at(W, 1); }
uint64_t blocked_states(int W) { return counts().at(W - 1, 1); }

bool needs_u64(int W) {
  // Every main or blocked rank and every intermediate index sum is < M.
  return main_states(W) > 0xffffffffull;
}

template <typename Idx>
void build_width_tables(int W, WidthTables<Idx> *t, int cap) {
  const CountTable &c = counts_capped(cap);
  memset(t, 0, sizeof(*t));
  for (int w = 0; w <= FDP_MAXW; ++w)
    for (int h = 0; h < FDP_HT; ++h) t->H[w][h] = Idx(c.H[w][h]);
  for (int pos = 0; pos < FDP_MAXW; ++pos)
    for (int h = 0; h < FDP_HT; ++h) {
      uint64_t t1 = c.at(pos, h), r1 = h > 0 ? c.at(pos, h - 1) : 0;
      uint64_t cR = c.at(pos + 1, h), cr1 = h > 0 ? c.at(pos + 1, h - 1) : 0;
      t->S[pos][h].t1 = Idx(t1);
      t->S[pos][h].t2 = Idx(t1 + r1);
      t->S[pos][h].cR = Idx(cR);
      t->S[pos][h].cL = Idx(cR + cr1);
    }
  // OFF[p][h][pair]: prefix sums of the pair sub-block sizes inside one high run.
  for (int p = 1; p < FDP_MAXW; ++p)
    for (int h = 0; h < FDP_HT; ++h) {
      uint64_t off = 0;
      for (int pr = 0; pr < PR_COUNT; ++pr) {
        t->OFF[p][h][pr] = Idx(off);
        int h1 = h + sym_delta(pair_first(pr));
        int h2 = h1 + sym_delta(pair_second(pr));
        if (h1 >= 0 && h2 >= 0 && h1 <= c.cap && h2 <= c.cap) off += c.at(p - 1, h2);
      }
    }
  (void)W;
}

template void build_width_tables<uint32_t>(int, WidthTables<uint32_t> *, int);
template void build_width_tables<uint64_t>(int, WidthTables<uint64_t> *, int);

static inline uint32_t mget(uint64_t m, int k) { return uint32_t(m >> (2 * k)) & 3u; }
static inline uint64_t msetpair(uint64_t m, int p, uint32_t v) {
  uint64_t z = 15ull << (2 * (p - 1));
  return (m & ~z) | (uint64_t(v) << (2 * (p - 1)));
}
static inline uint64_t mset(uint64_t m, int k, uint32_t v) {
  uint64_t z = 3ull << (2 * k);
  return (m & ~z) | (uint64_t(v) << (2 * k));
}
static inline uint64_t mshrink(uint64_t m, int k) {
  uint64_t mask = (1ull << (2 * k)) - 1;
  return ((m & ~mask) >> 2) | (m & mask);
}

uint64_t rank_word(uint64_t m, int width, int cap) {
  const CountTable &c = counts_capped(cap);
  uint64_t r = 0;
  int h = 1;
  for (int pos = width - 1; pos >= 0; --pos) {
    uint32_t s = mget(m, pos);
    if (s > SYM_N) r += c.at(pos, h);
    if (s > SYM_R && h > 0) r += c.at(pos, h - 1);
    if (s == SYM_R) --h;
    else if (s == SYM_L) ++h;
  }
  return r;
}

uint64_t unrank_word(uint64_t rank, int width, int cap) {
  const CountTable &c = counts_capped(cap);
  uint64_t m = 0;
  int h = 1;
  for (int pos = width - 1; pos >= 0; --pos) {
    uint64_t z = c.at(pos, h);
    if (rank < z) continue;
    rank -= z;
    if (h > 0) {
      z = c.at(pos, h - 1);
      if (rank < z) {
        m |= uint64_t(SYM_R) << (2 * pos);
        --h;
        continue;
      }
      rank -= z;
    }
    m |= uint64_t(SYM_L) << (2 * pos);
    ++h;
  }
  return m;
}

// Scalar closure scans (TR.hpp:66-103 semantics).
static int match_left(uint64_t t, int p) {
  int q = p - 1, s = 1;
  while (s) {
    if (--q < 0) return -1;
    uint32_t v = mget(t, q);
    if (v == SYM_L) ++s;
    else if (v == SYM_R) --s;
  }
  return q;
}
static int match_right(uint64_t t, int width, int p) {
  int q = p, s = 1;
  while (s) {
    if (++q >= width) return -1;
    uint32_t v = mget(t, q);
    if (v == SYM_L) --s;
    else if (v == SYM_R) ++s;
  }
  return q;
}

int include_horizontal(uint64_t m, int width, int p, uint64_t *out) {
  uint32_t pair = uint32_t(m >> (2 * (p - 1))) & 15u;
  uint64_t t;
  switch (pair) {
    case 0x0: *out = msetpair(m, p, 0x9); return 1;                  // NN -> LR
    case 0x1: case 0x2:                                               // NR, NL
      if (p == 1) { *out = msetpair(m, p, pair == 0x1 ? 0x4 : 0x8); return 1; }
      *out = mshrink(m, p); return 2;
    case 0x4: *out = msetpair(m, p, 0x1); return 1;                  // RN -> NR
    case 0x8: *out = msetpair(m, p, 0x2); return 1;                  // LN -> NL
    case 0xa: {                                                       // LL
      t = msetpair(m, p, 0);
      int q = match_left(t, p);
      if (q < 0) return 0;
      t = mset(t, q, SYM_L);
      if (p == 1) { *out = t; return 1; }
      *out = mshrink(t, p - 1); return 2;
    }
    case 0x5: {                                                       // RR
      t = msetpair(m, p, 0);
      int q = match_right(t, width, p);
      if (q < 0) return 0;
      t = mset(t, q, SYM_R);
      if (p == 1) { *out = t; return 1; }
      *out = mshrink(t, p - 1); return 2;
    }
    case 0x6:                                                         // RL
      t = msetpair(m, p, 0);
      if (p == 1) { *out = t; return 1; }
      *out = mshrink(t, p - 1); return 2;
    default: return 0;
  }
}

uint64_t first_row_state(uint64_t mask, int W) {
  uint64_t m = uint64_t(SYM_R) << (2 * (W - 1)), t = 0;
  for (int p = W - 1; p >= 1; --p)
    if ((mask >> (p - 1)) & 1u) {
      include_horizontal(m, W, p, &t);
      m = t;
    }
  return m;
}

// Prefix counts: words of `len` symbols from height 1 that end at height h,
// heights in [0, cap].
static void prefix_counts(int len, uint64_t *P /* FDP_HT */, int cap) {
  uint64_t Q[FDP_HT];
  for (int h = 0; h < FDP_HT; ++h) P[h] = 0;
  P[1] = 1;
  for (int i = 0; i < len; ++i) {
    for (int h = 0; h < FDP_HT; ++h) Q[h] = 0;
    for (int h = 0; h < FDP_HT; ++h) {
      if (!P[h]) continue;
      Q[h] += P[h];
      if (h > 0) Q[h - 1] += P[h];
      if (h + 1 < FDP_HT && h + 1 <= cap) Q[h + 1] += P[h];
    }
    for (int h = 0; h < FDP_HT; ++h) P[h] = Q[h];
  }
}

uint64_t cell_bytes(int W, int p, int cap) {
  // Minimum traffic of one cell of the in-place sweep, one modulus:
  //   reads : every main word (identity words are closure sources), and the
  //           blocked input except at p = W-1, where it is known to be zero;
  //   writes: main words whose value can change (pair LR/NR/NL or N at p;
  //           at p = 1 the pairs NN, LR, NR, RN) and the blocked output
  //           except at p = 1, which produces none.
  const CountTable &c = counts_capped(cap);
  uint64_t M = main_states_capped(W, cap), D = blocked_states_capped(W, cap), wm = 0;
  uint64_t P[FDP_HT];
  prefix_counts(W - 1 - p, P, c.cap);
  for (int h = 0; h < FDP_HT; ++h) {
    if (!P[h]) continue;
    const uint64_t lr = h + 1 <= c.cap ? c.at(p - 1, h) : 0;  // the LR sub-block
    if (p == 1)  // NN, LR (h = 0) and NR, RN (h = 1): one word each
      wm += P[h] * ((h == 0 ? 1 + lr : 0) + (h == 1 ? 2 : 0));
    else
      wm += P[h] * (c.at(p, h) + lr);
  }
  const uint64_t rd = M + (p < W - 1 ? D : 0);
  const uint64_t wr = wm + (p >= 2 ? D : 0);
  return 4 * (rd + wr);
}

uint64_t row_bytes(int W, int cap) {
  uint64_t b = 0;
  for (int p = W - 1; p >= 1; --p) b += cell_bytes(W, p, cap);
  return b;
}

uint64_t cell_transitions(int W, int cap) { return main_states_capped(W, cap) + blocked_states_capped(W, cap); }

std::vector<int> bounded_prefix_caps(int W) {
  std::vector<int> caps;
  const double full = double(main_states(W));
  for (int cap = 2; cap - 1 <= W - 2 && cap < FDP_HT - 2; ++cap) {
    if (double(main_states_capped(W, cap)) >= 0.95 * full) break;
    caps.push_back(cap);
  }
  return caps;
}

}  // namespace fdp
