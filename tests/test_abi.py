"""C ABI: the library loads, exports every declared entry point, and the pure
host planner returns the state sizes and byte model of the path.  CPU only."""
import ctypes
import os
import re

import pytest

import fdp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(fdp_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = fdp.lib()
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s


def test_version():
    assert b"sm_100a" in fdp.lib().fdp_version()


@pytest.mark.parametrize("n,M,D", [
    (18, 32652735, 11662902), (20, 258215664, 91695540), (22, 2062967382, 728997192),
    (23, 5850674704, 2062967382)])
def test_state_counts(n, M, D):
    # H_DP[W][1] / H_DP[W-1][1] as printed by the reference's PLAN_ONLY mode
    assert fdp.main_states(n + 1) == M and fdp.blocked_states(n + 1) == D
    pl = fdp.plan(n, [4294967291])
    assert pl.main_states == M and pl.blocked_states == D
    assert pl.state_bytes == 4 * (M + D) and pl.scratch_bytes == 0


def test_plan_n22_batched():
    pl = fdp.plan(22, list(range(4294967000, 4294967014)), lanes=14, budget=180 * 10**9)
    assert pl.lanes == 14 and pl.passes == 1 and pl.fits == 1
    assert abs(pl.state_bytes / 2**30 - 145.61) < 0.01
    assert pl.rows == 21 and pl.cells_per_row == 22 and pl.index_bits == 32
    assert fdp.plan(23, [7], lanes=1).index_bits == 64
    # 16 lanes at n=23 need 471.7 GiB: does not fit a B200
    assert fdp.plan(23, list(range(100, 116)), lanes=16, budget=180 * 10**9).fits == 0


def test_byte_model():
    W = 23
    row = sum(fdp.cell_bytes(W, p) for p in range(1, W))
    assert abs(row / 1e9 - 392.77) < 0.01
    M, D = fdp.main_states(W), fdp.blocked_states(W)
    # p = W-1: no blocked read; p = 1: no blocked write
    assert fdp.cell_bytes(W, W - 1) < 4 * (M + D) + 4 * (M + D)
    assert fdp.cell_bytes(W, 0) == 0 and fdp.cell_bytes(W, W) == 0


def test_plan_rejects_bad_problems():
    with pytest.raises(fdp.FdpError) as e:
        fdp.plan(0, [7])
    assert e.value.status == fdp.FDP_ERR_ARGS
    with pytest.raises(fdp.FdpError) as e:
        fdp.plan(10, [1])
    assert e.value.status == fdp.FDP_ERR_MODULUS
    with pytest.raises(fdp.FdpError):
        fdp.plan(10, [7], lanes=17)


def test_create_without_gpu_reports_gpu_count():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(fdp.FdpError) as e:
        fdp.Engine(0)
    assert e.value.status == fdp.FDP_ERR_GPU_COUNT


def test_lane_panels_and_spans():
    # Panels are greedy widths 8, 4, 2, 1; a span is consecutive panels holding
    # at most 8 lanes (the unit a cell launch of several spans splits into).
    import fdp
    for lanes in range(1, 17):
        panels = fdp.lane_panels(lanes)
        assert sum(w for _, w in panels) == lanes
        assert [w for _, w in panels] == sorted((w for _, w in panels), reverse=True)
        spans = fdp.lane_spans(lanes)
        assert spans[0][0] == 0 and spans[-1][1] == lanes
        assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
        assert all(0 < e - s <= 8 for s, e in spans)
        assert all(any(p == s for p, _ in panels) for s, _ in spans)  # spans start on a panel
    assert fdp.lane_spans(14) == [(0, 8), (8, 14)]
    assert fdp.lane_spans(8) == [(0, 8)] and fdp.lane_spans(6) == [(0, 6)]


def test_misaligned_panel_pointers_are_rejected_on_the_host():
    # An 8-lane panel word is one 256-bit access, so caller-owned state must be
    # aligned to one word of the widest panel.  The check runs before anything
    # that needs a context or a device: these pointers are never dereferenced.
    import ctypes
    lib = fdp.lib()
    apply_cells = lib.fdp_apply_cells
    noalloc = lib.fdp_first_row_dot_noalloc
    noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_uint32), ctypes.c_void_p,
                        ctypes.c_void_p, ctypes.c_void_p]
    noalloc.restype = ctypes.c_int

    def mods(k):
        return (ctypes.c_uint32 * k)(*([4294967291] * k))

    for lanes, main, blk in ((8, 0x10010, 0x10000), (14, 0x10000, 0x10010), (16, 0x10008, 0x10000),
                             (4, 0x10000, 0x10008), (7, 0x10004, 0x10000), (2, 0x10004, 0x10000)):
        assert apply_cells(None, 13, 12, 1, lanes, mods(lanes), main, blk, None) == fdp.FDP_ERR_ARGS
        assert b"aligned" in lib.fdp_last_error()
    for lanes, main in ((8, 0x10010), (16, 0x10008), (5, 0x10008), (3, 0x10004)):
        assert noalloc(13, lanes, mods(lanes), main, 0x20000, None) == fdp.FDP_ERR_ARGS
        assert b"aligned" in lib.fdp_last_error()
