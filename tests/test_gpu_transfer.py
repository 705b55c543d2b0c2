"""Operator variants against the oracle's forward recurrence: the CSR
transfer map (single cell and paired cells, as tests/factor_transfer_map_test.cu
and factor_transfer_batch_test.cu of the reference check at W=10) and the
two-cell pull (reverse2)."""
import numpy as np
import pytest

import fdp
import oracle_lib as orc

pytestmark = pytest.mark.gpu
MODS = [2, 4294967291, 4294966997]


def _case(width, lanes, seed):
    rng = np.random.default_rng(seed)
    M, D = orc.main_states(width), orc.main_states(width - 1)
    mods = [MODS[i % 3] for i in range(lanes)]
    main = np.stack([rng.integers(0, m, size=M, dtype=np.uint64) for m in mods], 1).astype(np.uint32)
    blk = np.stack([rng.integers(0, m, size=D, dtype=np.uint64) for m in mods], 1).astype(np.uint32)
    return M, D, mods, main, blk


def _want(width, cells, mods, main, blk):
    om, ob = main.copy(), blk.copy()
    for l, m in enumerate(mods):
        a, b = main[:, l].copy(), blk[:, l].copy()
        for p in cells:
            a, b = orc.forward_cell(width, p, m, a, b)
        om[:, l], ob[:, l] = a, b
    return om, ob


def _dev(a):
    import torch
    return torch.from_numpy(fdp.pack_lanes(a).view(np.int32)).cuda()


def _run(apply, M, D, mods, main, blk):
    import torch
    im, ib = _dev(main), _dev(blk)
    om = torch.zeros_like(im)
    ob = torch.zeros_like(ib)
    apply(im.data_ptr(), ib.data_ptr(), om.data_ptr(), ob.data_ptr())
    torch.cuda.synchronize()
    # inputs are untouched (out of place)
    assert np.array_equal(fdp.unpack_lanes(im.cpu().numpy().view(np.uint32), M, len(mods)), main)
    return (fdp.unpack_lanes(om.cpu().numpy().view(np.uint32), M, len(mods)),
            fdp.unpack_lanes(ob.cpu().numpy().view(np.uint32), D, len(mods)))


@pytest.mark.parametrize("width", [4, 7, 10])
@pytest.mark.parametrize("paired", [False, True])
def test_transfer_map_matches_forward(engine, width, paired):
    for p in range(width - 1, 1 if paired else 0, -1):
        M, D, mods, main, blk = _case(width, 3, 100 * width + p)
        tm = engine.transfer_map(width, p, paired)
        info = tm.info()
        assert info["rows"] == M + D and info["edges"] > 0
        got = _run(lambda a, b, c, d: tm.apply(mods, a, b, c, d), M, D, mods, main, blk)
        want = _want(width, [p, p - 1] if paired else [p], mods, main, blk)
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])
        tm.close()


@pytest.mark.parametrize("width,lanes", [(6, 1), (9, 8), (11, 3)])
def test_reverse2_matches_two_cells(engine, width, lanes):
    for p in range(width - 1, 1, -1):
        M, D, mods, main, blk = _case(width, lanes, 7 * width + p)
        got = _run(lambda a, b, c, d: engine.reverse2_apply(width, p, mods, a, b, c, d), M, D, mods, main, blk)
        want = _want(width, [p, p - 1], mods, main, blk)
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])


def test_transfer_map_lane_panels(engine):
    width, p = 12, 7
    M, D, mods, main, blk = _case(width, 14, 5)
    tm = engine.transfer_map(width, p, paired=True)
    got = _run(lambda a, b, c, d: tm.apply(mods, a, b, c, d), M, D, mods, main, blk)
    want = _want(width, [p, p - 1], mods, main, blk)
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])


@pytest.mark.parametrize("width,p,paired,fixed,occupied", [
    (10, 6, False, 4, 2), (10, 7, True, 5, 3), (10, 3, False, 2, 1), (10, 4, True, 2, 0),
    (14, 9, True, 6, 3), (14, 5, False, 4, 4), (14, 8, False, 7, 2)])
def test_factor_map_groups_match_forward(engine, width, p, paired, fixed, occupied):
    # One CSR built on the representative group, applied to every conjugate
    # group (all masks with `occupied` of the bottom `fixed` positions set, up
    # to 32 per call): each written row equals the forward recurrence of the
    # whole vector, and the groups' rows are written exactly once.
    import itertools
    import torch
    mod = 4294967291
    masks = [sum(1 << q for q in c) for c in itertools.combinations(range(fixed), occupied)][:32]
    rng = np.random.default_rng(1000 * width + 10 * p + fixed)
    M, D = orc.main_states(width), orc.main_states(width - 1)
    main = rng.integers(0, mod, size=M, dtype=np.uint64).astype(np.uint32)
    blk = rng.integers(0, mod, size=D, dtype=np.uint64).astype(np.uint32)
    cells = [p, p - 1] if paired else [p]
    wm, wb = main.copy(), blk.copy()
    for q in cells:
        wm, wb = orc.forward_cell(width, q, mod, wm, wb)
    fm = engine.factor_map(width, p, fixed, occupied, paired=paired)
    info = fm.info()
    assert info["group_main"] > 0 and info["edges"] > 0
    im = torch.from_numpy(main.view(np.int32)).cuda()
    ib = torch.from_numpy(blk.view(np.int32)).cuda()
    om = torch.full_like(im, -1)
    ob = torch.full_like(ib, -1)
    phases = fm.apply(mod, masks, im.data_ptr(), ib.data_ptr(), om.data_ptr(), ob.data_ptr(), timed=True)
    torch.cuda.synchronize()
    assert len(phases) == 3 and all(t >= 0 for t in phases)
    assert np.array_equal(im.cpu().numpy().view(np.uint32), main)
    gm = om.cpu().numpy().view(np.uint32)
    gb = ob.cpu().numpy().view(np.uint32)
    hit_m, hit_b = gm != 0xFFFFFFFF, gb != 0xFFFFFFFF
    assert hit_m.sum() == len(masks) * info["group_main"]
    assert hit_b.sum() == len(masks) * info["group_blocked"]
    np.testing.assert_array_equal(gm[hit_m], wm[hit_m])
    np.testing.assert_array_equal(gb[hit_b], wb[hit_b])
    fm.close()


def test_factor_map_rejects_a_group_the_cells_touch(engine):
    with pytest.raises(fdp.FdpError):
        engine.factor_map(10, 4, 4, 2)               # fixed > p - 1
    with pytest.raises(fdp.FdpError):
        engine.factor_map(10, 4, 3, 1, paired=True)  # fixed > p - 2
    fm = engine.factor_map(10, 6, 4, 2, max_groups=2)
    import torch
    z = torch.zeros(8, dtype=torch.int32, device="cuda")
    with pytest.raises(fdp.FdpError):  # a mask with the wrong number of set bits
        fm.apply(4294967291, [0b111], z.data_ptr(), z.data_ptr(), z.data_ptr(), z.data_ptr())
    with pytest.raises(fdp.FdpError):  # more groups than the arena holds
        fm.apply(4294967291, [3, 5, 6], z.data_ptr(), z.data_ptr(), z.data_ptr(), z.data_ptr())
    fm.close()
