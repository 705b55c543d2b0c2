// Host-compiled check of the sm_100a kernels' own item logic (fdp_item.cuh,
// fdp_core.cuh are host+device) against the oracle's forward recurrence.
// Test infrastructure: built and run by tests/test_host_kernel_logic.py.
//
//   cells  : every cell p of widths 2..Wmax, lane counts 1/3/7/8/14/16 (32-
//            and 64-bit indices), random residues under moduli {2, 4294967291,
//            4294966997}; items visited in warp chunks of 32..256 with the
//            shared prefix decode, in index order or in the grouped order of
//            the small-p kernel path (every c = R/L item, then the c = N items
//            backwards), exactly as the kernel may schedule them; the first
//            cell of a row also with a blocked input known to be zero.
//   capped : the same in the height-bounded spaces (caps 1..4): input supported
//            on the capped space, full-space oracle operator, projection back.
//   expand : the walk that moves a vector between spaces
//            (expand_step) against unrank in one space and rank in the other.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "fdp_host.h"
#include "fdp_item.cuh"

extern "C" int oracle_forward_cell(int, int, uint32_t, const uint32_t *, const uint32_t *, uint32_t *, uint32_t *);

using namespace fdp;

// Word of lane l of state s in the panel layout (greedy 8/4/2/1 panels).
static size_t lane_word(int K, size_t N, size_t s, int l) {
  for (int L0 = 0;;) {
    const int PW = K - L0 >= 8 ? 8 : K - L0 >= 4 ? 4 : (K - L0 >= 2 ? 2 : 1);
    if (l < L0 + PW) return size_t(L0) * N + s * PW + size_t(l - L0);
    L0 += PW;
  }
}

template <typename Idx, int K>
static int run_cells(int W, int cap, uint64_t seed) {
  static WidthTables<Idx> T;
  build_width_tables<Idx>(W, &T, cap);
  static CellSmem<Idx> sm;
  const bool full = cap >= FDP_FULL_CAP;
  const uint64_t Mf = main_states(W), Df = blocked_states(W);
  const uint64_t M = full ? Mf : main_states_capped(W, cap), D = full ? Df : blocked_states_capped(W, cap);
  std::mt19937_64 rng(seed);
  const uint32_t mods[3] = {2u, 4294967291u, 4294966997u};
  std::vector<Idx> cand(FDP_MAX_CAND);
  // Capped-space index -> full-space rank (identity in the full space).
  std::vector<uint64_t> fm(M), fb(D);
  for (uint64_t i = 0; i < M; ++i) fm[i] = full ? i : rank_word(unrank_word(i, W, cap), W);
  for (uint64_t i = 0; i < D; ++i) fb[i] = full ? i : rank_word(unrank_word(i, W - 1, cap), W - 1);
  int bad = 0;
  for (int p = W - 1; p >= 1; --p) {
    for (int x = 0; x <= FDP_MAXW; ++x)
      for (int y = 0; y < FDP_HS; ++y) sm.H[x][y] = T.H[x][y];
    for (int x = 0; x < FDP_MAXW; ++x)
      for (int y = 0; y < FDP_HS; ++y) sm.S[x][y] = T.S[x][y];
    for (int y = 0; y < FDP_HS; ++y)
      for (int z = 0; z < PR_COUNT; ++z) sm.OFF[y][z] = T.OFF[p][y][z];
    CellArgs a{};
    a.W = W;
    a.p = p;
    a.items = D;
    a.mstates = M;
    a.blk_in_zero = (p == W - 1 && (seed & 2)) ? 1 : 0;
    a.blk_out_p1 = 1;
    a.cap = cap;
    for (int k = 0; k < K; ++k) a.mod[k] = mods[(k + p) % 3];
    std::vector<uint32_t> mi(M * K), bi(D * K);
    for (uint64_t i = 0; i < M; ++i)
      for (int k = 0; k < K; ++k) mi[lane_word(K, M, i, k)] = uint32_t(rng() % a.mod[k]);
    for (uint64_t i = 0; i < D; ++i)
      for (int k = 0; k < K; ++k) bi[lane_word(K, D, i, k)] = a.blk_in_zero ? 0u : uint32_t(rng() % a.mod[k]);
    std::vector<uint32_t> gm = mi, gb = bi;
    a.main = gm.data();
    a.blk = gb.data();
    const uint64_t CH = uint64_t(32) * (1 + (seed + uint64_t(p)) % 8);
    const int mode = int((seed + uint64_t(p)) % 3);  // 0: no sharing; 1: shared, index order; 2: shared, grouped
    for (uint64_t jb = 0; jb < D; jb += CH) {
      const uint64_t jl = std::min(D, jb + CH) - 1;
      const Prefix<Idx> pf = mode ? shared_prefix<Idx>(a, sm, Idx(jb), Idx(jl)) : empty_prefix<Idx>(a);
      if (mode < 2) {
        for (uint64_t j = jb; j <= jl; ++j) cell_item<Idx, K>(a, sm, Idx(j), pf, cand.data(), 1);
      } else {
        std::vector<Head<Idx>> hx, hn;
        for (uint64_t j = jb; j <= jl; ++j) {
          const Head<Idx> hd = decode_head<Idx>(a, sm, Idx(j), pf);
          (hd.c ? hx : hn).push_back(hd);
        }
        for (const auto &hd : hx) item_x<Idx, K>(a, sm, hd);
        for (size_t k = hn.size(); k-- > 0;) item_n<Idx, K>(a, sm, hn[k], cand.data(), 1);
      }
    }
    for (int k = 0; k < K; ++k) {
      std::vector<uint32_t> m1(Mf, 0), b1(Df, 0), m2(Mf), b2(Df);
      for (uint64_t i = 0; i < M; ++i) m1[fm[i]] = mi[lane_word(K, M, i, k)];
      for (uint64_t i = 0; i < D; ++i) b1[fb[i]] = bi[lane_word(K, D, i, k)];
      oracle_forward_cell(W, p, a.mod[k], m1.data(), b1.data(), m2.data(), b2.data());
      for (uint64_t i = 0; i < M; ++i)
        if (gm[lane_word(K, M, i, k)] != m2[fm[i]]) {
          if (bad < 5) printf("K=%d W=%d cap=%d p=%d lane %d main %llu\n", K, W, cap, p, k, (unsigned long long)i);
          ++bad;
        }
      for (uint64_t i = 0; i < D; ++i)
        if (gb[lane_word(K, D, i, k)] != b2[fb[i]]) {
          if (bad < 5) printf("K=%d W=%d cap=%d p=%d lane %d blocked %llu\n", K, W, cap, p, k, (unsigned long long)i);
          ++bad;
        }
    }
  }
  return bad;
}

static int run_expand(int W, int cf, int ct) {
  const CountTable &F = counts_capped(cf), &T = counts_capped(ct);
  const uint64_t Nf = main_states_capped(W, cf);
  int bad = 0;
  for (uint64_t lo : {uint64_t(0), Nf / 3}) {
    const uint64_t n = Nf - lo;
    for (uint64_t cb = 0; cb < n; cb += 256) {
      const uint64_t ce = std::min(n, cb + 256);
      uint64_t r0 = lo + cb, r1 = lo + ce - 1, j0 = 0;
      int h = 1, pos = W - 1;
      for (; pos >= 0; --pos) {  // the chunk's shared top symbols, as the kernel walks them
        uint64_t a0 = r0, a1 = r1, jj = j0, b1 = 0;
        int h0 = h, h1 = h;
        expand_step(F.H, T.H, pos, a0, jj, h0);
        expand_step(F.H, T.H, pos, a1, b1, h1);
        if (h0 != h1) break;
        r0 = a0;
        r1 = a1;
        j0 = jj;
        h = h0;
      }
      const uint64_t sub = lo + cb - r0;
      for (uint64_t i = cb; i < ce; ++i) {
        uint64_t r = lo + i - sub, j = j0;
        int hh = h;
        for (int q = pos; q >= 0; --q) expand_step(F.H, T.H, q, r, j, hh);
        if (j != rank_word(unrank_word(lo + i, W, cf), W, ct)) {
          if (bad < 5) printf("expand W=%d %d->%d index %llu\n", W, cf, ct, (unsigned long long)(lo + i));
          ++bad;
        }
      }
    }
  }
  return bad;
}

int main(int argc, char **argv) {
  const int wmax = argc > 1 ? atoi(argv[1]) : 11;
  const int wcap = argc > 2 ? atoi(argv[2]) : 10;
  int bad = 0;
  for (int W = 2; W <= wmax; ++W) {
    bad += run_cells<uint32_t, 1>(W, FDP_FULL_CAP, uint64_t(W));
    bad += run_cells<uint64_t, 3>(W, FDP_FULL_CAP, 100u + W);
    bad += run_cells<uint32_t, 7>(W, FDP_FULL_CAP, 200u + W);
    bad += run_cells<uint32_t, 8>(W, FDP_FULL_CAP, 300u + W);
    bad += run_cells<uint32_t, 14>(W, FDP_FULL_CAP, 400u + W);
    bad += run_cells<uint64_t, 16>(W, FDP_FULL_CAP, 500u + W);
  }
  printf("cells bad=%d\n", bad);
  for (int W = 3; W <= wcap; ++W)
    for (int cap = 1; cap <= 4; ++cap) {
      bad += run_cells<uint32_t, 1>(W, cap, uint64_t(7 * W + cap));
      bad += run_cells<uint32_t, 14>(W, cap, uint64_t(11 * W + cap));
      bad += run_cells<uint64_t, 3>(W, cap, uint64_t(13 * W + cap));
    }
  printf("capped bad=%d\n", bad);
  for (int W = 3; W <= wmax + 1; ++W)
    for (int cf = 1; cf <= 5; ++cf) {
      bad += run_expand(W, cf, cf + 1);
      bad += run_expand(W, cf, FDP_FULL_CAP);
    }
  printf("bad=%d\n", bad);
  return bad != 0;
}
