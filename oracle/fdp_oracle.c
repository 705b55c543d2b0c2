/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's CPU semantics for the Grid-FP
 * frontier transition.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference leg may load this library, and only as the checker
 * or the timed CPU baseline.  The product (libfdp.so) never links or calls it.
 *
 * Parity pins (checked by tests/test_oracle_golden.py):
 *   - exact path counts n=1..9 (scripts/test/golden_cpu.py:9-19),
 *   - known residues n=9 mod 4294967291 / 4294966997
 *     (scripts/test/groupbatch-runtime.py:17),
 *   - the reverse-test witness chain (tests/gridfp_reverse_test.cpp:24-37),
 *   - agreement with the reference's own CPU counter (third_party/ggcount,
 *     built unmodified into oracle/_ref by oracle/Makefile) for n<=14,
 *   - a brute-force DFS over simple paths for n<=6.
 *
 * Restated algorithm (forward, push form):
 *   - MateID words of 2-bit symbols N=0,R=1,L=2 (src/common/gridfp_transition.hpp:20-33);
 *   - include_horizontal / closure matching / blocked_exclude
 *     (src/common/gridfp_transition.hpp:66-146);
 *   - the per-cell forward recurrence over every legal word
 *     (tests/groupbatch_operator_test.cu:127-146);
 *   - path-count DP and canonical rank (GB.cu:172 build_full_dp, GB.cu:1568 rank_full,
 *     GB.cu = src/cuda/b300/oneesan_cuda_gridfp_b300_hbm32_factorized_fullprerank_orbit_blockfused_groupbatch_batch.cu);
 *   - first-row initialiser and first-row dot product (GB.cu:1081-1116).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define OR_MAXW 28
#define OR_N 0
#define OR_R 1
#define OR_L 2

typedef uint64_t mate_t;

static uint64_t HDP[OR_MAXW + 1][OR_MAXW + 3];
static int hdp_ready = 0;

/* GB.cu:172 build_full_dp: Motzkin-path counts from height h down to 0. */
static void build_dp(void) {
    if (hdp_ready) return;
    memset(HDP, 0, sizeof(HDP));
    HDP[0][0] = 1;
    for (int w = 1; w <= OR_MAXW; ++w)
        for (int h = 0; h <= OR_MAXW + 1; ++h) {
            uint64_t x = HDP[w - 1][h];
            if (h > 0) x += HDP[w - 1][h - 1];
            if (h + 1 <= OR_MAXW + 1) x += HDP[w - 1][h + 1];
            HDP[w][h] = x;
        }
    hdp_ready = 1;
}

uint64_t oracle_hdp(int w, int h) {
    build_dp();
    if (w < 0 || w > OR_MAXW || h < 0 || h > OR_MAXW + 1) return 0;
    return HDP[w][h];
}

/* TR.hpp:28-33 symbol accessors */
static inline int mget(mate_t m, int k) { return (int)((m >> (2 * k)) & 3u); }
static inline int mpair(mate_t m, int p) { return (int)((m >> (2 * (p - 1))) & 15u); }
static inline mate_t mset(mate_t m, int k, int v) {
    mate_t z = (mate_t)3 << (2 * k);
    return (m & ~z) | ((mate_t)v << (2 * k));
}
static inline mate_t msetpair(mate_t m, int p, int v) {
    mate_t z = (mate_t)15 << (2 * (p - 1));
    return (m & ~z) | ((mate_t)v << (2 * (p - 1)));
}
static inline mate_t mshrink(mate_t m, int k) {
    mate_t mask = ((mate_t)1 << (2 * k)) - 1;
    return ((m & ~mask) >> 2) | (m & mask);
}
static inline mate_t minsert(mate_t m, int k, int v) {
    mate_t lowmask = k ? (((mate_t)1 << (2 * k)) - 1) : 0;
    return (m & lowmask) | ((mate_t)v << (2 * k)) | ((m & ~lowmask) << 2);
}

/* TR.hpp:66-103, scalar form of the closure scans. */
static int match_left(mate_t t, int p) {
    int q = p - 1, s = 1;
    while (s) {
        --q;
        if (q < 0) return -1;
        int v = mget(t, q);
        if (v == OR_L) ++s; else if (v == OR_R) --s;
    }
    return q;
}
static int match_right(mate_t t, int width, int p) {
    int q = p, s = 1;
    while (s) {
        ++q;
        if (q >= width) return -1;
        int v = mget(t, q);
        if (v == OR_L) --s; else if (v == OR_R) ++s;
    }
    return q;
}

enum { P_NN = 0x0, P_NR = 0x1, P_NL = 0x2, P_RN = 0x4, P_RR = 0x5, P_RL = 0x6,
       P_LN = 0x8, P_LR = 0x9, P_LL = 0xa };

/* TR.hpp:113-144 include_horizontal.  Returns 0 if invalid, else 1 (main) or 2 (blocked). */
int oracle_include(mate_t m, int width, int p, mate_t *out) {
    mate_t t;
    int pair = mpair(m, p);
    switch (pair) {
    case P_NN: *out = msetpair(m, p, P_LR); return 1;
    case P_NR: case P_NL:
        if (p == 1) { *out = msetpair(m, p, pair == P_NR ? P_RN : P_LN); return 1; }
        *out = mshrink(m, p); return 2;
    case P_RN: *out = msetpair(m, p, P_NR); return 1;
    case P_LN: *out = msetpair(m, p, P_NL); return 1;
    case P_LL: {
        t = msetpair(m, p, P_NN);
        int q = match_left(t, p);
        if (q < 0) return 0;
        t = mset(t, q, OR_L);
        if (p == 1) { *out = t; return 1; }
        *out = mshrink(t, p - 1); return 2;
    }
    case P_RR: {
        t = msetpair(m, p, P_NN);
        int q = match_right(t, width, p);
        if (q < 0) return 0;
        t = mset(t, q, OR_R);
        if (p == 1) { *out = t; return 1; }
        *out = mshrink(t, p - 1); return 2;
    }
    case P_RL:
        t = msetpair(m, p, P_NN);
        if (p == 1) { *out = t; return 1; }
        *out = mshrink(t, p - 1); return 2;
    default:
        return 0;
    }
}

/* GB.cu:1568 rank_full: lexicographic rank (N<R<L) among words starting at height 1. */
uint64_t oracle_rank(mate_t m, int width) {
    build_dp();
    uint64_t r = 0;
    int h = 1;
    for (int pos = width - 1; pos >= 0; --pos) {
        int s = mget(m, pos);
        if (s > OR_N) r += HDP[pos][h];
        if (s > OR_R && h > 0) r += HDP[pos][h - 1];
        if (s == OR_R) --h; else if (s == OR_L) ++h;
    }
    return r;
}

mate_t oracle_unrank(uint64_t rank, int width) {
    build_dp();
    mate_t m = 0;
    int h = 1;
    for (int pos = width - 1; pos >= 0; --pos) {
        uint64_t z = HDP[pos][h];
        if (rank < z) continue;
        rank -= z;
        if (h > 0) {
            z = HDP[pos][h - 1];
            if (rank < z) { m |= (mate_t)OR_R << (2 * pos); --h; continue; }
            rank -= z;
        }
        m |= (mate_t)OR_L << (2 * pos);
        ++h;
    }
    return m;
}

uint64_t oracle_main_states(int width) { build_dp(); return HDP[width][1]; }

static inline uint32_t addm(uint32_t a, uint32_t b, uint32_t mod) {
    return (uint32_t)(((uint64_t)a + b) % mod);
}

/*
 * One cell of the forward recurrence (tests/groupbatch_operator_test.cu:127-146):
 *   main_out  = main_in + sum_{m: include(m,p) main}   main_in[m]
 *                       + sum_{b}                     block_in[b] at blocked_exclude(b,p)
 *   block_out =           sum_{m: include(m,p) blocked} main_in[m]
 * Vectors are in canonical rank order, each entry in [0, mod).
 */
int oracle_forward_cell(int width, int p, uint32_t mod, const uint32_t *main_in,
                        const uint32_t *block_in, uint32_t *main_out, uint32_t *block_out) {
    build_dp();
    if (width < 2 || width > OR_MAXW || p < 1 || p >= width || mod < 2) return -1;
    uint64_t M = HDP[width][1], D = HDP[width - 1][1];
    memcpy(main_out, main_in, (size_t)M * sizeof(uint32_t));
    memset(block_out, 0, (size_t)D * sizeof(uint32_t));
    for (uint64_t i = 0; i < M; ++i) {
        mate_t w = oracle_unrank(i, width), t;
        int kind = oracle_include(w, width, p, &t);
        if (!kind) continue;
        uint32_t v = main_in[i];
        if (kind == 2) {
            uint64_t j = oracle_rank(t, width - 1);
            block_out[j] = addm(block_out[j], v, mod);
        } else {
            uint64_t j = oracle_rank(t, width);
            main_out[j] = addm(main_out[j], v, mod);
        }
    }
    for (uint64_t b = 0; b < D; ++b) {
        mate_t w = oracle_unrank(b, width - 1);
        uint64_t j = oracle_rank(minsert(w, p, OR_N), width);
        main_out[j] = addm(main_out[j], block_in[b], mod);
    }
    return 0;
}

/* GB.cu:1081-1096: the state reached by one first-row edge mask. */
mate_t oracle_first_row_state(uint64_t mask, int width) {
    mate_t m = (mate_t)OR_R << (2 * (width - 1)), t;
    for (int p = width - 1; p >= 1; --p)
        if ((mask >> (p - 1)) & 1u) {
            oracle_include(m, width, p, &t);
            m = t;
        }
    return m;
}

/*
 * Full residue: row-0 initialiser, rows 1..W-2 of cells p=W-1..1, then the
 * first-row dot product (GB.cu:2218-2256 with prefixK=1).
 * Returns 0 on success.
 */
int oracle_residue(int n, uint32_t mod, uint32_t *out) {
    build_dp();
    int W = n + 1;
    if (n < 1 || W > OR_MAXW || mod < 2) return -1;
    uint64_t M = HDP[W][1], D = HDP[W - 1][1];
    uint32_t *a = calloc(M, 4), *b = calloc(D ? D : 1, 4), *a2 = calloc(M, 4), *b2 = calloc(D ? D : 1, 4);
    if (!a || !b || !a2 || !b2) { free(a); free(b); free(a2); free(b2); return -2; }
    uint64_t total = (uint64_t)1 << (W - 1);
    for (uint64_t mask = 0; mask < total; ++mask)
        a[oracle_rank(oracle_first_row_state(mask, W), W)] = 1 % mod;
    for (int row = 1; row < W - 1; ++row)
        for (int p = W - 1; p >= 1; --p) {
            oracle_forward_cell(W, p, mod, a, b, a2, b2);
            uint32_t *t = a; a = a2; a2 = t;
            t = b; b = b2; b2 = t;
        }
    uint64_t acc = 0;
    for (uint64_t mask = 0; mask < total; ++mask) {
        acc += a[oracle_rank(oracle_first_row_state(mask, W), W)];
        acc %= mod;
    }
    *out = (uint32_t)acc;
    free(a); free(b); free(a2); free(b2);
    return 0;
}

/*
 * Brute-force DFS: simple paths from corner (0,0) to (n,n) on the
 * (n+1)x(n+1) vertex grid (README.md:3).  Independent of the frontier DP.
 */
typedef struct { int v; uint64_t seen; } dfs_task;
typedef struct {
    const dfs_task *tasks; int ntasks, side, next_shared;
    uint64_t count;
} dfs_job;

static uint64_t dfs(int side, int v, uint64_t seen) {
    if (v == side * side - 1) return 1;
    uint64_t n = 0;
    int r = v / side, c = v % side;
    if (r > 0 && !((seen >> (v - side)) & 1)) n += dfs(side, v - side, seen | ((uint64_t)1 << (v - side)));
    if (r + 1 < side && !((seen >> (v + side)) & 1)) n += dfs(side, v + side, seen | ((uint64_t)1 << (v + side)));
    if (c > 0 && !((seen >> (v - 1)) & 1)) n += dfs(side, v - 1, seen | ((uint64_t)1 << (v - 1)));
    if (c + 1 < side && !((seen >> (v + 1)) & 1)) n += dfs(side, v + 1, seen | ((uint64_t)1 << (v + 1)));
    return n;
}

/* Expand the search tree to a fixed depth; each partial path is an independent task. */
static void dfs_expand(int side, int v, uint64_t seen, int depth, dfs_task *out, int *n, int cap,
                       uint64_t *done) {
    if (v == side * side - 1) { ++*done; return; }
    if (depth == 0) { if (*n < cap) { out[*n].v = v; out[*n].seen = seen; } ++*n; return; }
    int r = v / side, c = v % side;
    int nb[4], k = 0;
    if (r > 0) nb[k++] = v - side;
    if (r + 1 < side) nb[k++] = v + side;
    if (c > 0) nb[k++] = v - 1;
    if (c + 1 < side) nb[k++] = v + 1;
    for (int i = 0; i < k; ++i)
        if (!((seen >> nb[i]) & 1))
            dfs_expand(side, nb[i], seen | ((uint64_t)1 << nb[i]), depth - 1, out, n, cap, done);
}

static pthread_mutex_t dfs_lock = PTHREAD_MUTEX_INITIALIZER;
static void *dfs_worker(void *arg) {
    dfs_job *job = (dfs_job *)arg;
    uint64_t local = 0;
    for (;;) {
        pthread_mutex_lock(&dfs_lock);
        int t = job->next_shared++;
        pthread_mutex_unlock(&dfs_lock);
        if (t >= job->ntasks) break;
        local += dfs(job->side, job->tasks[t].v, job->tasks[t].seen);
    }
    pthread_mutex_lock(&dfs_lock);
    job->count += local;
    pthread_mutex_unlock(&dfs_lock);
    return NULL;
}

uint64_t oracle_dfs_count(int n, int threads) {
    if (n < 1 || n > 6) return 0;
    int side = n + 1, cap = 1 << 16, ntasks = 0;
    uint64_t done = 0;
    dfs_task *tasks = malloc(sizeof(dfs_task) * cap);
    if (!tasks) return 0;
    dfs_expand(side, 0, 1, n >= 5 ? 12 : 2, tasks, &ntasks, cap, &done);
    if (ntasks > cap) { free(tasks); return 0; }
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    dfs_job job = {tasks, ntasks, side, 0, done};
    pthread_t th[256];
    for (int i = 0; i < threads; ++i) pthread_create(&th[i], NULL, dfs_worker, &job);
    for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
    free(tasks);
    return job.count;
}
