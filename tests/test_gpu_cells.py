"""Cell-operator parity: the sm_100a pull kernel (through the C ABI) against the
oracle's forward recurrence, full vectors, bit-exact.

Mirrors tests/groupbatch_operator_test.cu of the reference: random coefficients
mod {2, 4294967291, 4294966997} (:101), every single cell including p=1 and the
two forced windows (:104-119), several lane counts and two replays (:147-157),
full-vector compare (:172).
"""
import numpy as np
import pytest

import oracle_lib as orc

pytestmark = pytest.mark.gpu

MODS = [2, 4294967291, 4294966997]


def _rand(rng, n, lanes, mods):
    a = np.empty((n, lanes), dtype=np.uint64)
    for l in range(lanes):
        a[:, l] = rng.integers(0, mods[l], size=n, dtype=np.uint64)
    return a.astype(np.uint32)


def _device(a):
    import torch
    import fdp
    return torch.from_numpy(fdp.pack_lanes(a).view(np.int32)).cuda()


def _host(t, n, lanes):
    import fdp
    return fdp.unpack_lanes(t.cpu().numpy().view(np.uint32), n, lanes)


def _oracle_window(width, p_hi, p_lo, mods, main, block):
    lanes = len(mods)
    mo, bo = main.copy(), block.copy()
    for l in range(lanes):
        m, b = main[:, l].copy(), block[:, l].copy()
        for p in range(p_hi, p_lo - 1, -1):
            m, b = orc.forward_cell(width, p, mods[l], m, b)
        mo[:, l], bo[:, l] = m, b
    return mo, bo


def _run(engine, width, p_hi, p_lo, mods, seed, replays=1):
    import torch
    rng = np.random.default_rng(seed)
    M, D = orc.main_states(width), orc.main_states(width - 1)
    main = _rand(rng, M, len(mods), mods)
    block = _rand(rng, D, len(mods), mods)
    want_m, want_b = _oracle_window(width, p_hi, p_lo, mods, main, block)
    for _ in range(replays):
        dm, db = _device(main), _device(block)
        engine.apply_cells(width, p_hi, p_lo, mods, dm.data_ptr(), db.data_ptr())
        torch.cuda.synchronize()
        got_m, got_b = _host(dm, M, len(mods)), _host(db, D, len(mods))
        np.testing.assert_array_equal(got_m, want_m)
        np.testing.assert_array_equal(got_b, want_b)


@pytest.mark.parametrize("width", list(range(2, 13)))
@pytest.mark.parametrize("lanes", [1, 3, 4])
def test_every_single_cell(engine, width, lanes):
    for p in range(width - 1, 0, -1):
        mods = [MODS[(i + p) % 3] for i in range(lanes)]
        _run(engine, width, p, p, mods, seed=1000 * width + 10 * p + lanes)


@pytest.mark.parametrize("width", [10, 14])
def test_forced_windows_all_lane_counts(engine, width):
    low = width // 2
    for lanes in range(1, 17):
        mods = [MODS[i % 3] for i in range(lanes)]
        for (hi, lo) in ((width - 1, low + 1), (low, 1), (width - 1, 1)):
            _run(engine, width, hi, lo, mods, seed=77 * lanes + hi, replays=2 if lanes in (1, 16) else 1)


def test_same_modulus_lanes_are_independent_vectors(engine):
    # GROUPBATCH lane semantics: L independent vectors under one modulus.
    _run(engine, 11, 10, 1, [4294967291] * 8, seed=5)


def test_zero_input_stays_zero(engine):
    import torch
    width = 9
    M, D = orc.main_states(width), orc.main_states(width - 1)
    dm = torch.zeros(M * 2, dtype=torch.int32, device="cuda")
    db = torch.zeros(D * 2, dtype=torch.int32, device="cuda")
    engine.apply_cells(width, width - 1, 1, [4294967291, 2], dm.data_ptr(), db.data_ptr())
    torch.cuda.synchronize()
    assert int(dm.abs().sum()) == 0 and int(db.abs().sum()) == 0


def test_tuning_never_changes_results(engine):
    # block size, grid size, panel splitting, warp-chunk size, prefix
    # sharing, grouping (per chunk or with carry-over queues) and span
    # splitting are performance knobs only
    try:
        for block, grid, split, items, share, compact, citems, spans, carry in (
                (128, 0, True, 1, 99, -1, 4, 1, -1), (64, 37, False, 7, 1, 30, 3, 1000, -1),
                (256, 1, True, 64, 1, 5, 1, 4, 1), (96, 0, False, 3, 5, 1, 2, 1, -1),
                (256, 0, False, 1, 1, 30, 4, 6, 1), (160, 3, False, 4, 2, 30, 4, 9, -1),
                (256, 0, False, 8, 4, 30, 16, 1000, 1), (64, 5, False, 2, 2, 30, 8, 1000, 1),
                (224, 0, True, 5, 3, 30, 1, 1000, 1)):
            engine.set_tuning(block=block, grid=grid, split_panels=split, lane_items=items, share_min=share,
                              compact_max_p=compact, compact_items=citems, split_spans_min_p=spans,
                              compact_carry=carry)
            assert engine.get_tuning() == {"block": block, "grid": grid, "split_panels": split,
                                           "bounded_prefix": True, "lane_items": items, "share_min": share,
                                           "compact_max_p": compact, "compact_items": citems,
                                           "row_init_rows": 0, "row_init_product": 0, "split_spans_min_p": spans,
                                           "compact_carry": carry}
            _run(engine, 12, 11, 1, [MODS[i % 3] for i in range(14)], seed=block + grid)
            _run(engine, 12, 3, 1, [MODS[i % 3] for i in range(8)], seed=block + items)
            _run(engine, 12, 5, 1, [MODS[i % 3] for i in range(5)], seed=block + citems)
    finally:
        engine.set_tuning()


def test_tuning_rejects_bad_block(engine):
    import fdp
    with pytest.raises(fdp.FdpError):
        engine.set_tuning(block=100)
    with pytest.raises(fdp.FdpError):
        engine.set_tuning(block=512)
