"""End-to-end residues through the C ABI (fdp_run_sync) against the oracle, the
reference's published residues and exact counts reconstructed by CRT."""
import pytest

import oracle_lib as orc

pytestmark = pytest.mark.gpu

P = orc.largest_primes_below_2_32(48)
GOLDEN = {1: 2, 2: 12, 3: 184, 4: 8512, 5: 1262816, 6: 575780564, 7: 789360053252,
          8: 3266598486981642, 9: 41044208702632496804}  # scripts/test/golden_cpu.py:9-19

# Residues published by the reference for its GPU solvers.
KNOWN = [
    (9, 4294967291, 2674633373), (9, 4294966997, 3332982389),    # scripts/test/groupbatch-runtime.py:17
    (18, 4294967291, 503411004),                                 # docs/results/reverse-algorithm-2026-09-05.md:53
    (16, 2147483647, 1234504449), (17, 2147483647, 1667553532),  # docs/b300-hbm32.md:479-481
    (18, 2147483647, 624312750),
    (20, 4294967291, 2308006916), (20, 4294966997, 3704549185),  # scripts/test/groupbatch-scratch.py:17
    (21, 4294966997, 2124618149), (21, 4294967291, 998035516),   # scripts/run/autotune.py:28, docs/b300-hbm32.md:554
    (22, 4294967291, 1245069298),  # docs/results/groupbatch-interleaved-2026-09-05.json:1027, 1291
]


@pytest.mark.parametrize("n", list(range(1, 12)))
def test_residues_match_oracle_plain_and_batched(engine, n):
    mods = [P[0], P[10], 2, 3]
    want = [orc.residue(n, m) for m in mods]
    assert engine.residues(n, mods, lanes=1).residues == want
    assert engine.residues(n, mods, lanes=4).residues == want


def test_exact_counts_by_crt(engine):
    for n, exact in GOLDEN.items():
        mods = P[:3]
        res = engine.residues(n, mods, lanes=3).residues
        x, m = orc.crt(dict(zip(mods, res)))
        assert m > exact and x == exact, n


@pytest.mark.parametrize("n,mod,want", KNOWN)
def test_published_residues(engine, n, mod, want):
    assert engine.residues(n, [mod], lanes=1).residues == [want]


def test_lane_counts_agree(engine):
    # Above 8 lanes a pass sweeps its two lane spans as concurrent launch
    # chains: 9 = {0-7} + {8}, 14 = {0-7} + {8-13}, 16 = {0-7} + {8-15}.
    n = 13
    mods = P[:16]
    plain = engine.residues(n, mods, lanes=1).residues
    for lanes in (2, 5, 7, 9, 14, 16):
        assert engine.residues(n, mods, lanes=lanes).residues == plain
    assert plain[0] == orc.residue(n, mods[0])


def test_several_grid_sizes_in_one_graph(engine):
    problems = [(9, P[:3]), (14, P[3:7]), (12, [2, 3, 5]), (17, P[:14]), (6, [P[0]])]
    got, st = engine.residues_multi(problems)
    for (n, mods), res in zip(problems, got):
        assert res == engine.residues(n, mods, lanes=1).residues
    assert got[0][:1] == [2674633373] and st.kernel_launches > 0 and st.device_s > 0


def test_passes_in_one_graph(engine):
    mods = P[:20] + [2, 3]
    got = engine.residues(12, mods, lanes=8)  # 3 passes, one graph launch
    assert got.residues == engine.residues(12, mods, lanes=1).residues
    assert got.residues[:2] == [orc.residue(12, mods[0]), orc.residue(12, mods[1])]


def test_autotune_picks_a_correct_configuration(engine):
    mods = P[:6]
    try:
        rec = engine.autotune(14, mods, max_lanes=6, repeats=1)
        best = rec["best"]
        # no published residue at n = 14: the check runs at n = 9
        assert rec["known_residue_check"] == {"n": 9, "status": "ok"}
        assert 1 <= best["lanes"] <= 6 and best["s_per_residue"] > 0
        tuned = engine.get_tuning()
        for knob in ("block", "lane_items", "share_min", "compact_max_p", "compact_items"):
            assert tuned[knob] == best[knob], knob
        assert {c["lanes"] for c in rec["candidates"]} >= {1, 2, 4, 6}
        assert engine.residues(14, mods, lanes=best["lanes"]).residues == [orc.residue(14, m) for m in mods[:1]] + \
            engine.residues(14, mods[1:], lanes=1).residues
    finally:
        engine.set_tuning()


def test_autotune_checks_the_published_residue_of_its_own_n(engine):
    # n = 18 has a published residue mod 4294967291 (503411004): the tuned
    # configuration is checked at n = 18 itself; stage 2 tried the knobs.
    try:
        rec = engine.autotune(18, P[:4], max_lanes=4, repeats=1)
        assert rec["known_residue_check"] == {"n": 18, "status": "ok"}
        knobs = {k for c in rec["candidates"] for k in c if k in ("lane_items", "share_min", "compact_max_p",
                                                                 "compact_items")}
        assert knobs == {"lane_items", "share_min", "compact_max_p", "compact_items"}
        lanes = rec["best"]["lanes"]
        assert engine.residues(18, P[:4], lanes=lanes).residues == [503411004, 2737033518, 2864590416, 278648965]
    finally:
        engine.set_tuning()


def test_bounded_prefix_equals_full_rows(engine):
    try:
        for n, mods in ((4, P[:1]), (9, P[:2]), (15, P[:5]), (16, P[:14])):
            engine.set_tuning(bounded_prefix=False, row_init_rows=-1)
            full = engine.residues(n, mods, lanes=len(mods)).residues
            engine.set_tuning(bounded_prefix=True, row_init_rows=-1)
            assert engine.residues(n, mods, lanes=len(mods)).residues == full, n
            assert engine.residues(n, mods, lanes=1).residues == full, n
    finally:
        engine.set_tuning()


@pytest.mark.parametrize("product", [0, 1], ids=["tensor-cores", "cuda-cores"])
@pytest.mark.parametrize("rows", [2, 3, 4, 5, 6, 7])
def test_row_init_equals_row_sweeps(engine, rows, product):
    """The row-k initialiser (the state after the first `rows` rows of
    vertices, computed by the column automaton) gives the residues of the row
    sweeps, in the bounded and the full space, for every lane count kind, with
    its products on the tensor cores (8-bit limbs) and on the CUDA cores."""
    try:
        for n, mods, lanes in ((6, P[:2], 2), (9, [2, 3, P[0]], 3), (12, P[:8], 8), (14, P[:14], 14), (15, P[:3], 1),
                               (17, [P[0], 2147483647], 2)):
            engine.set_tuning(row_init_rows=-1)
            want = engine.residues(n, mods, lanes=lanes).residues
            for bounded in (True, False):
                engine.set_tuning(bounded_prefix=bounded, row_init_rows=rows, row_init_product=product)
                assert engine.residues(n, mods, lanes=lanes).residues == want, (n, rows, bounded)
    finally:
        engine.set_tuning()
