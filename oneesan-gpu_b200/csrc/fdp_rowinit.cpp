// Row-k initialiser, host side: the column automaton and the fill plan
// (fdp_rowinit.h).
#include "fdp_rowinit.h"

#include <algorithm>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <unordered_map>

#include "fdp_host.h"

namespace fdp {
namespace {

constexpr int kMaxRows = 7;
enum { SN = 0, SR = 1, SL = 2 };  // word symbols

// Slot codes of a cut: 0 none, 1 + k open arc k, 16 + i closing pair i, 32 + i U-turn i.
inline bool is_open(int c) { return c >= 1 && c < 16; }
inline bool is_close(int c) { return c >= 16 && c < 32; }
inline bool is_uturn(int c) { return c >= 32; }

uint64_t key_of(const int *s, int R) {
  uint64_t k = 0;
  for (int i = 0; i < R; ++i) k |= uint64_t(uint8_t(s[i])) << (8 * i);
  return k;
}

void unkey(uint64_t k, int R, int *s) {
  for (int i = 0; i < R; ++i) s[i] = int((k >> (8 * i)) & 0xffu);
}

// Renumber closing pairs and U-turns in order of first appearance.
void canonicalise(int *s, int R) {
  int cmap[64], umap[64], nc = 0, nu = 0;
  for (int i = 0; i < 64; ++i) cmap[i] = umap[i] = -1;
  for (int i = 0; i < R; ++i) {
    if (is_close(s[i])) {
      int &m = cmap[s[i] - 16];
      if (m < 0) m = nc++;
      s[i] = 16 + m;
    } else if (is_uturn(s[i])) {
      int &m = umap[s[i] - 32];
      if (m < 0) m = nu++;
      s[i] = 32 + m;
    }
  }
}

struct UF {
  int p[2 * kMaxRows + 2];
  void init(int n) {
    for (int i = 0; i < n; ++i) p[i] = i;
  }
  int find(int x) {
    while (p[x] != x) x = p[x] = p[p[x]];
    return x;
  }
  bool unite(int a, int b) {  // false: already joined (a cycle)
    a = find(a);
    b = find(b);
    if (a == b) return false;
    p[a] = b;
    return true;
  }
};

enum EndKind { E_OUT, E_D, E_START, E_OPEN, E_CPART };
struct End {
  int kind, v;
};

// All cuts reachable from `in_slots` (nullptr: the initial state before the
// first column) by one column reading `sym`, with their numbers of column edge
// sets.  The column's vertices are rows 0..R-1; its edges are the vertical
// edges between consecutive rows, the down edge below row R-1 (present iff
// sym != N) and, unless this is the last column, one outgoing horizontal edge
// per row.
void column_step(const int *in_slots, int R, int sym, bool first, bool last, std::map<uint64_t, uint32_t> &out) {
  int slots[kMaxRows] = {0};
  int h = 1;  // the start corner's open arc
  if (!first) {
    h = 0;
    for (int i = 0; i < R; ++i) {
      slots[i] = in_slots[i];
      if (is_open(slots[i])) ++h;
    }
  }
  const int d = sym == SN ? 0 : 1;
  if (sym == SR && h == 0) return;
  // Union-find elements: vertices 0..R-1, then one element per incoming piece
  // (an open arc's piece, a U-turn, or each of the two pieces of a closing pair).
  int piece[kMaxRows], pkind[2 * kMaxRows + 2], pgroup[2 * kMaxRows + 2];
  int nel = R;
  {
    int uel[64];
    for (int i = 0; i < 64; ++i) uel[i] = -1;
    for (int i = 0; i < R; ++i) {
      piece[i] = -1;
      if (!slots[i]) continue;
      if (is_uturn(slots[i])) {
        int &e = uel[slots[i] - 32];
        if (e < 0) {
          e = nel++;
          pkind[e] = 'U';
          pgroup[e] = slots[i] - 32;
        }
        piece[i] = e;
      } else {
        piece[i] = nel++;
        pkind[piece[i]] = is_open(slots[i]) ? 'O' : 'C';
        pgroup[piece[i]] = is_open(slots[i]) ? slots[i] - 1 : slots[i] - 16;
      }
    }
  }
  const int nv = R - 1, nh = last ? 0 : R;
  for (uint32_t bits = 0; bits < (1u << (nv + nh)); ++bits) {
    int e[kMaxRows] = {0}, hh[kMaxRows] = {0};
    for (int i = 0; i < nv; ++i) e[i] = (bits >> i) & 1u;
    for (int i = 0; i < nh; ++i) hh[i] = (bits >> (nv + i)) & 1u;
    bool ok = true;
    for (int i = 0; i < R && ok; ++i) {
      const int deg = (slots[i] != 0) + hh[i] + (i > 0 ? e[i - 1] : 0) + (i < nv ? e[i] : 0) + (i == R - 1 ? d : 0);
      if (first && i == 0) ok = deg == 1;  // the start corner
      else ok = deg == 0 || deg == 2;
    }
    if (!ok) continue;
    UF uf;
    uf.init(nel);
    for (int i = 0; i < R && ok; ++i)
      if (piece[i] >= 0 && !uf.unite(i, piece[i])) ok = false;
    for (int i = 0; i < nv && ok; ++i)
      if (e[i] && !uf.unite(i, i + 1)) ok = false;
    if (!ok) continue;
    // The ends of every joined set (each must be a path: exactly two ends).
    End ends[2 * kMaxRows + 2][3];
    int nend[2 * kMaxRows + 2] = {0};
    auto add_end = [&](int root, int kind, int v) {
      if (nend[root] < 3) ends[root][nend[root]] = End{kind, v};
      ++nend[root];
    };
    for (int i = 0; i < R; ++i)
      if (hh[i]) add_end(uf.find(i), E_OUT, i);
    if (d) add_end(uf.find(R - 1), E_D, 0);
    if (first) add_end(uf.find(0), E_START, 0);
    for (int el = R; el < nel; ++el) {
      if (pkind[el] == 'O') add_end(uf.find(el), E_OPEN, pgroup[el]);
      else if (pkind[el] == 'C') add_end(uf.find(el), E_CPART, pgroup[el]);
    }
    int nw[kMaxRows] = {0};
    int cont_open[kMaxRows + 1];  // open arc -> its new slot
    for (int k = 0; k <= kMaxRows; ++k) cont_open[k] = -1;
    int cslots[64][2], ncs[64] = {0};
    bool cdone[64] = {false};
    int next_u = 0, dkind = -1, dval = -1;
    for (int root = 0; root < nel && ok; ++root) {
      if (!nend[root]) continue;
      if (nend[root] != 2) {
        ok = false;
        break;
      }
      End a = ends[root][0], b = ends[root][1];
      if (a.kind > b.kind) std::swap(a, b);
      if (a.kind == E_OUT && b.kind == E_OUT) {  // a new U-turn
        nw[a.v] = nw[b.v] = 32 + next_u;
        ++next_u;
      } else if (a.kind == E_OUT && b.kind == E_OPEN) {  // an open arc goes on
        cont_open[b.v] = a.v;
      } else if (a.kind == E_OUT && b.kind == E_CPART) {  // half of a closing pair goes on
        if (ncs[b.v] >= 2) ok = false;
        else cslots[b.v][ncs[b.v]++] = a.v;
      } else if (a.kind == E_OUT && b.kind == E_START) {  // the start corner's arc goes on
        cont_open[0] = a.v;
      } else if (a.kind == E_OUT && b.kind == E_D) {  // the down edge's piece goes on
        dkind = E_OUT;
        dval = a.v;
      } else if (a.kind == E_D && b.kind == E_OPEN) {  // the down edge closes an open arc here
        dkind = E_OPEN;
        dval = b.v;
      } else if (a.kind == E_D && b.kind == E_START) {  // the start corner's arc goes down here
        dkind = E_START;
      } else if (a.kind == E_CPART && b.kind == E_CPART && a.v == b.v) {  // a closing pair meets
        cdone[a.v] = true;
      } else {
        ok = false;
      }
    }
    if (!ok) continue;
    int next_c = 0;
    for (int g = 0; g < 64 && ok; ++g) {
      if (!ncs[g]) continue;
      if (ncs[g] != 2 || cdone[g]) {
        ok = false;
        break;
      }
      nw[cslots[g][0]] = nw[cslots[g][1]] = 16 + next_c;
      ++next_c;
    }
    if (!ok) continue;
    int newh = h;
    if (sym == SL) {
      if (dkind != E_OUT) continue;
      cont_open[h] = dval;
      newh = h + 1;
    } else if (sym == SR) {
      const int top = h - 1;
      if (dkind == E_OPEN) {
        if (dval != top) continue;
        newh = h - 1;
      } else if (dkind == E_START) {
        if (h != 1) continue;
        newh = 0;
      } else if (dkind == E_OUT) {
        if (cont_open[top] < 0) continue;
        nw[cont_open[top]] = nw[dval] = 16 + next_c;
        ++next_c;
        cont_open[top] = -1;
        newh = h - 1;
      } else {
        continue;
      }
    }
    // Every arc still open goes on with exactly one slot.
    bool fine = true;
    for (int k = 0; k <= kMaxRows; ++k)
      if ((cont_open[k] >= 0) != (k < newh)) fine = false;
    if (!fine) continue;
    for (int k = 0; k < newh; ++k) nw[cont_open[k]] = 1 + k;
    canonicalise(nw, R);
    out[key_of(nw, R)] += 1;
  }
}

RowAutomaton build(int R) {
  if (R < 1 || R > kMaxRows) throw std::invalid_argument("row automaton: rows must be 1..7");
  RowAutomaton a;
  a.rows = R;
  std::unordered_map<uint64_t, int> id;
  std::vector<uint64_t> keys;
  std::deque<int> todo;
  auto get = [&](uint64_t k) {
    auto it = id.find(k);
    if (it != id.end()) return it->second;
    const int n = int(keys.size());
    id.emplace(k, n);
    keys.push_back(k);
    todo.push_back(n);
    return n;
  };
  for (int sym = 0; sym < 3; ++sym) {
    std::map<uint64_t, uint32_t> out;
    column_step(nullptr, R, sym, true, false, out);
    for (auto &kv : out) a.first[sym].push_back(AutTrans{-1, get(kv.first), kv.second});
  }
  while (!todo.empty()) {
    const int s = todo.front();
    todo.pop_front();
    int slots[kMaxRows];
    unkey(keys[size_t(s)], R, slots);
    for (int sym = 0; sym < 3; ++sym) {
      std::map<uint64_t, uint32_t> out;
      column_step(slots, R, sym, false, false, out);
      for (auto &kv : out) a.inner[sym].push_back(AutTrans{s, get(kv.first), kv.second});
      std::map<uint64_t, uint32_t> fin;
      column_step(slots, R, sym, false, true, fin);
      for (auto &kv : fin) {
        if (kv.first != 0) throw std::logic_error("row automaton: the last column left a cut");
        a.last[sym].push_back(AutTrans{s, -1, kv.second});
      }
    }
  }
  a.nstates = int(keys.size());
  a.height.resize(size_t(a.nstates));
  a.index.resize(size_t(a.nstates));
  a.per_height.assign(size_t(R) + 1, 0);
  for (int s = 0; s < a.nstates; ++s) {
    int slots[kMaxRows], h = 0;
    unkey(keys[size_t(s)], R, slots);
    for (int i = 0; i < R; ++i) h += is_open(slots[i]) ? 1 : 0;
    a.height[size_t(s)] = h;
    a.index[size_t(s)] = a.per_height[size_t(h)]++;
  }
  return a;
}

}  // namespace

const RowAutomaton &row_automaton(int rows) {
  static std::mutex mu;
  static std::map<int, std::unique_ptr<RowAutomaton>> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(rows);
  if (it == cache.end()) it = cache.emplace(rows, std::make_unique<RowAutomaton>(build(rows))).first;
  return *it->second;
}

uint32_t row_automaton_coeff(const RowAutomaton &a, uint64_t word, int W, uint32_t mod) {
  std::vector<uint64_t> v(size_t(a.nstates), 0), nv(size_t(a.nstates));
  auto sym_at = [&](int pos) { return int((word >> (2 * pos)) & 3u); };
  for (const AutTrans &t : a.first[sym_at(W - 1)]) v[size_t(t.to)] = (v[size_t(t.to)] + t.weight) % mod;
  for (int pos = W - 2; pos >= 1; --pos) {
    std::fill(nv.begin(), nv.end(), 0);
    for (const AutTrans &t : a.inner[sym_at(pos)])
      if (v[size_t(t.from)]) nv[size_t(t.to)] = (nv[size_t(t.to)] + v[size_t(t.from)] * t.weight) % mod;
    v.swap(nv);
  }
  uint64_t c = 0;
  for (const AutTrans &t : a.last[sym_at(0)]) c = (c + v[size_t(t.from)] * t.weight) % mod;
  return uint32_t(c);
}

RowInitPlan plan_row_init(int W, int rows, int cap) {
  const RowAutomaton &a = row_automaton(rows);
  const CountTable &H = counts_capped(cap);
  RowInitPlan pl;
  pl.W = W;
  pl.rows = rows;
  pl.cap = cap;
  pl.states = H.H[W][1];
  pl.K = a.per_height;
  const int hmax = std::min(rows, cap);
  pl.hmax = hmax;
  auto completable = [&](int k, int h) { return h >= 0 && h <= hmax && H.H[W - k][h] > 0; };
  // cnt[k][h]: prefixes of k symbols ending at height h (heights in 0..hmax, completable)
  std::vector<std::vector<uint64_t>> cnt(size_t(W), std::vector<uint64_t>(size_t(hmax) + 2, 0));
  cnt[0][1] = completable(0, 1) ? 1 : 0;
  for (int k = 1; k < W; ++k)
    for (int h = 0; h <= hmax; ++h) {
      if (!completable(k, h)) continue;
      uint64_t c = cnt[size_t(k - 1)][size_t(h)];
      if (h + 1 <= hmax) c += cnt[size_t(k - 1)][size_t(h + 1)];  // R from h+1
      if (h >= 1) c += cnt[size_t(k - 1)][size_t(h - 1)];         // L from h-1
      cnt[size_t(k)][size_t(h)] = c;
    }
  uint64_t best = ~0ull;
  for (int P = 1; P < W; ++P) {
    uint64_t mac = 0;
    for (int h = 0; h <= hmax; ++h) mac += cnt[size_t(P)][size_t(h)] * H.H[W - P][h] * uint64_t(a.per_height[size_t(h)]);
    if (mac < best) {
      best = mac;
      pl.P = P;
    }
  }
  pl.S = W - pl.P;
  pl.mac = best;
  // Prefix trie in canonical order (the children of a node in N, R, L order).
  pl.parent.resize(size_t(pl.P));
  pl.sym.resize(size_t(pl.P));
  pl.height.resize(size_t(pl.P));
  pl.row.resize(size_t(pl.P));
  pl.rows_of.assign(size_t(pl.P), std::vector<uint64_t>(size_t(rows) + 1, 0));
  std::vector<uint64_t> base_prev{0}, base_cur;
  std::vector<int> h_prev{1};
  for (int k = 1; k <= pl.P; ++k) {
    const int pos = W - k;  // position of the k-th symbol
    auto &par = pl.parent[size_t(k - 1)];
    auto &sy = pl.sym[size_t(k - 1)];
    auto &hh = pl.height[size_t(k - 1)];
    auto &rw = pl.row[size_t(k - 1)];
    auto &nof = pl.rows_of[size_t(k - 1)];
    base_cur.clear();
    for (size_t i = 0; i < h_prev.size(); ++i) {
      const int h = h_prev[i];
      for (int s = 0; s < 3; ++s) {
        const int h2 = s == SN ? h : (s == SR ? h - 1 : h + 1);
        if (!completable(k, h2)) continue;
        uint64_t b = base_prev[i];
        if (s >= SR) b += H.H[pos][h];
        if (s == SL && h > 0) b += H.H[pos][h - 1];
        par.push_back(k == 1 ? -1 : int32_t(i));
        sy.push_back(uint8_t(s));
        hh.push_back(uint8_t(h2));
        rw.push_back(int32_t(nof[size_t(h2)]++));
        base_cur.push_back(b);
      }
    }
    base_prev = base_cur;
    h_prev.assign(hh.begin(), hh.end());
  }
  pl.base = base_prev;
  pl.C.assign(size_t(pl.S) + 1, std::vector<uint64_t>(size_t(hmax) + 2, 0));
  for (int k = 0; k <= pl.S; ++k)
    for (int g = 0; g <= hmax; ++g) pl.C[size_t(k)][size_t(g)] = H.H[k][g];
  return pl;
}

uint64_t row_init_table_bytes(const RowInitPlan &pl) {
  const RowAutomaton &a = row_automaton(pl.rows);
  uint64_t b = 0;
  // Automaton: state ids, first-column edges (3 + 1 offsets, targets and
  // weights), interior edges both ways (3 x (states + 1) offsets each, one
  // index and one weight per edge), last-column weights (3 x states).
  uint64_t inner = 0, first = 0;
  for (int s = 0; s < 3; ++s) {
    inner += a.inner[s].size();
    first += a.first[s].size();
  }
  b += 4 * uint64_t(a.nstates) + 4 * 4 + 8 * first + 2 * (12 * uint64_t(a.nstates + 1) + 8 * inner) +
       12 * uint64_t(a.nstates);
  // Prefix trie: parent and row (4 bytes each), symbol and height (1 byte
  // each) per prefix of every level, and the last level's state bases.
  uint64_t prefixes = 0;
  for (int k = 0; k < pl.P; ++k) prefixes += pl.parent[size_t(k)].size();
  b += 10 * prefixes;
  if (pl.P > 0) b += 8 * pl.parent[size_t(pl.P - 1)].size();
  return b;
}

uint64_t row_init_scratch_words(const RowInitPlan &pl) {
  uint64_t pre = 0, suf = 0;
  for (int k = 0; k < pl.P; ++k) {
    uint64_t w = 0;
    for (int h = 0; h <= pl.hmax; ++h) w += pl.rows_of[size_t(k)][size_t(h)] * uint64_t(pl.K[size_t(h)]);
    pre = std::max(pre, w);
  }
  for (int k = 1; k <= pl.S; ++k) {
    uint64_t w = 0;
    for (int g = 0; g <= pl.hmax; ++g) w += pl.C[size_t(k)][size_t(g)] * uint64_t(pl.K[size_t(g)]);
    suf = std::max(suf, w);
  }
  // The tensor-core product's packed limb tiles of one height at a time:
  // 128-row A tiles of 16 KB and 64-row B tiles of 8 KB per 32-wide K step.
  uint64_t packed = 0;
  for (int h = 0; h <= pl.hmax; ++h) {
    const uint64_t K = uint64_t(pl.K[size_t(h)]), nks = (K + 31) / 32;
    const uint64_t rows = pl.rows_of[size_t(pl.P - 1)][size_t(h)], cols = pl.C[size_t(pl.S)][size_t(h)];
    if (!K || !rows || !cols) continue;
    packed = std::max(packed, ((rows + 127) / 128) * nks * 4096 + ((cols + 63) / 64) * nks * 2048);
  }
  return 2 * ((pre + 3) & ~uint64_t(3)) + 2 * ((suf + 3) & ~uint64_t(3)) + packed;
}

std::vector<uint32_t> row_init_fill_host(const RowInitPlan &pl, uint32_t mod) {
  const RowAutomaton &a = row_automaton(pl.rows);
  const int hmax = pl.hmax;
  std::vector<uint32_t> out(size_t(pl.states), 0);
  auto local = [&](int s) { return size_t(a.index[size_t(s)]); };
  // Prefix vectors, level by level (each over the states of its end height).
  std::vector<std::vector<uint64_t>> v_prev, v_cur;
  for (int k = 1; k <= pl.P; ++k) {
    const auto &par = pl.parent[size_t(k - 1)];
    const auto &sy = pl.sym[size_t(k - 1)];
    const auto &hh = pl.height[size_t(k - 1)];
    v_cur.assign(par.size(), {});
    for (size_t i = 0; i < par.size(); ++i) {
      std::vector<uint64_t> v(size_t(a.per_height[hh[i]]), 0);
      if (k == 1) {
        for (const AutTrans &t : a.first[sy[i]])
          if (a.height[size_t(t.to)] == hh[i]) v[local(t.to)] = (v[local(t.to)] + t.weight) % mod;
      } else {
        const auto &pv = v_prev[size_t(par[i])];
        const int hp = pl.height[size_t(k - 2)][size_t(par[i])];
        for (const AutTrans &t : a.inner[sy[i]]) {
          if (a.height[size_t(t.from)] != hp) continue;
          const uint64_t x = pv[local(t.from)];
          if (x) v[local(t.to)] = (v[local(t.to)] + x * t.weight) % mod;
        }
      }
      v_cur[i] = std::move(v);
    }
    v_prev.swap(v_cur);
  }
  // Suffix vectors: U[g] holds C[k][g] columns of K_g entries.
  std::vector<std::vector<uint64_t>> U(size_t(hmax) + 1), Un(size_t(hmax) + 1);
  for (int g = 0; g <= hmax; ++g) {
    const size_t Kg = size_t(a.per_height[size_t(g)]);
    U[size_t(g)].assign(Kg * pl.C[1][size_t(g)], 0);
    if (pl.C[1][size_t(g)] == 0) continue;  // one position left: N from 0 or R from 1
    const int sy = g == 0 ? SN : SR;
    for (const AutTrans &t : a.last[sy])
      if (a.height[size_t(t.from)] == g) U[size_t(g)][local(t.from)] = (U[size_t(g)][local(t.from)] + t.weight) % mod;
  }
  for (int k = 2; k <= pl.S; ++k) {
    for (int g = 0; g <= hmax; ++g) {
      const size_t Kg = size_t(a.per_height[size_t(g)]);
      const uint64_t Ck = pl.C[size_t(k)][size_t(g)];
      auto &dst = Un[size_t(g)];
      dst.assign(Kg * Ck, 0);
      for (uint64_t j = 0; j < Ck; ++j) {
        int sy, gc;
        uint64_t jc = j;
        if (jc < pl.C[size_t(k - 1)][size_t(g)]) {
          sy = SN;
          gc = g;
        } else {
          jc -= pl.C[size_t(k - 1)][size_t(g)];
          const uint64_t cr = g >= 1 ? pl.C[size_t(k - 1)][size_t(g - 1)] : 0;
          if (jc < cr) {
            sy = SR;
            gc = g - 1;
          } else {
            jc -= cr;
            sy = SL;
            gc = g + 1;
          }
        }
        if (gc > hmax) continue;  // passes above the strip's height: zero
        const size_t Kc = size_t(a.per_height[size_t(gc)]);
        const uint64_t *child = U[size_t(gc)].data() + jc * Kc;
        uint64_t *col = dst.data() + j * Kg;
        for (const AutTrans &t : a.inner[sy]) {
          if (a.height[size_t(t.from)] != g) continue;
          const uint64_t x = child[local(t.to)];
          if (x) col[local(t.from)] = (col[local(t.from)] + x * t.weight) % mod;
        }
      }
    }
    U.swap(Un);
  }
  // The products.
  const auto &htop = pl.height[size_t(pl.P - 1)];
  for (size_t i = 0; i < pl.base.size(); ++i) {
    const int h = htop[i];
    const size_t Kh = size_t(a.per_height[size_t(h)]);
    const uint64_t Ch = pl.C[size_t(pl.S)][size_t(h)];
    for (uint64_t j = 0; j < Ch; ++j) {
      uint64_t acc = 0;
      for (size_t q = 0; q < Kh; ++q) acc = (acc + v_prev[i][q] * U[size_t(h)][j * Kh + q]) % mod;
      out[size_t(pl.base[i] + j)] = uint32_t(acc);
    }
  }
  return out;
}

}  // namespace fdp
