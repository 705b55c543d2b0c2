"""Pins the oracle (the checker) to the reference's golden vectors and to the
reference's own CPU counter.  CPU only."""
import pytest

import oracle_lib as orc

# scripts/test/golden_cpu.py:9-19
GOLDEN = {1: 2, 2: 12, 3: 184, 4: 8512, 5: 1262816, 6: 575780564, 7: 789360053252,
          8: 3266598486981642, 9: 41044208702632496804}
P = orc.largest_primes_below_2_32(48)


def test_prime_table_matches_reference_head():
    # scripts/solve/path_bound.py:5-18, first row and the 11th entry
    assert P[:4] == [4294967291, 4294967279, 4294967231, 4294967197]
    assert P[10] == 4294966997 and P[-1] == 4294966087


@pytest.mark.parametrize("n", sorted(GOLDEN))
def test_oracle_exact_counts_by_crt(n):
    mods = P[:3]
    x, m = orc.crt({p: orc.residue(n, p) for p in mods})
    assert m > GOLDEN[n] and x == GOLDEN[n]


def test_oracle_published_residues():
    # scripts/test/groupbatch-runtime.py:17
    assert orc.residue(9, 4294967291) == 2674633373
    assert orc.residue(9, 4294966997) == 3332982389


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6])
def test_bruteforce_dfs(n):
    assert orc.dfs_count(n) == GOLDEN[n]


def test_reverse_witness_chain():
    # tests/gridfp_reverse_test.cpp:24-37: LLLRRRRN reaches the first-row support
    w, blocked = 43348, False
    for p in range(7, 0, -1):
        if blocked:
            # blocked_exclude = insert N at p
            lo = w & ((1 << (2 * p)) - 1)
            w = lo | ((w >> (2 * p)) << (2 * p + 2))
            blocked = False
        elif p in (4, 2):
            kind, w = orc.include(w, 8, p)
            assert kind
            blocked = kind == 2
    kind, support = orc.include(1 << 14, 8, 6)
    assert not blocked and w == support == 25600


def test_rank_unrank_roundtrip():
    for width in range(1, 12):
        for r in range(orc.main_states(width)):
            assert orc.rank(orc.unrank(r, width), width) == r


@pytest.mark.skipif(not orc.ggcount_available(), reason="reference counter not built (oracle/_ref)")
@pytest.mark.parametrize("n", [2, 5, 8, 11, 12])
def test_oracle_matches_reference_cpu_counter(n):
    for mod in (4294967291, 4294966997, 2147483647):
        assert orc.residue(n, mod) == orc.ggcount_residue(n, mod)
