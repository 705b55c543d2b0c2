"""fdp_first_row_dot_noalloc: residues read out of a caller-owned state with no
device allocation inside the library.

It serves callers that cannot call cudaMalloc because their own pool allocator
already holds the device memory (a serving HBM budget, a framework's caching
allocator) or because they must not take the device synchronisation that
cudaMalloc / cudaFree can cause.  The test builds the final state of an n=12
residue pass in buffers it owns, through the existing operator entry point
(fdp_apply_cells), reads the residues out with the no-allocation entry point
twice in a row, and requires both reads to equal the residues of the existing
entry point fdp_run_sync bit for bit (residues are exact integers).

This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import fdp
import oracle_lib as orc

pytestmark = pytest.mark.gpu


def noalloc(width, moduli, main_ptr, residues_ptr, stream=0):
    f = fdp.lib().fdp_first_row_dot_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_uint32), ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    mods = (ctypes.c_uint32 * len(moduli))(*moduli)
    return f(width, len(moduli), mods, main_ptr, residues_ptr, stream)


def test_noalloc_matches_run_sync_on_two_calls(engine):
    import torch
    n, moduli = 12, [4294967291, 4294966997, 2147483647]
    W, lanes = n + 1, len(moduli)
    M, D = fdp.main_states(W), fdp.blocked_states(W)

    # Row-0 state (every first-row state has coefficient 1), built on the host.
    init = np.zeros((M, lanes), dtype=np.uint32)
    for mask in range(1 << (W - 1)):
        init[orc.rank(int(orc.lib().oracle_first_row_state(mask, W)), W), :] = 1
    dm = torch.from_numpy(fdp.pack_lanes(init).view(np.int32)).cuda()
    db = torch.zeros(D * lanes, dtype=torch.int32, device="cuda")
    for _row in range(1, W - 1):
        engine.apply_cells(W, W - 1, 1, moduli, dm.data_ptr(), db.data_ptr())
    torch.cuda.synchronize()

    want = engine.residues(n, moduli, lanes=lanes).residues
    assert want == [orc.residue(n, m) for m in moduli]

    for _call in range(2):
        out = torch.full((lanes,), -1, dtype=torch.int32, device="cuda")
        assert noalloc(W, moduli, dm.data_ptr(), out.data_ptr()) == fdp.FDP_OK
        torch.cuda.synchronize()
        got = [int(x) for x in out.cpu().numpy().view(np.uint32)]
        assert got == want


def _final_state(engine, n, moduli, stream=0):
    """The final state of an n residue pass, in caller-owned torch buffers,
    built through fdp_apply_cells on `stream` (a cudaStream_t, 0: the engine's)."""
    import torch
    W, lanes = n + 1, len(moduli)
    M, D = fdp.main_states(W), fdp.blocked_states(W)
    init = np.zeros((M, lanes), dtype=np.uint32)
    for mask in range(1 << (W - 1)):
        init[orc.rank(int(orc.lib().oracle_first_row_state(mask, W)), W), :] = 1
    dm = torch.from_numpy(fdp.pack_lanes(init).view(np.int32)).cuda()
    db = torch.zeros(D * lanes, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    for _row in range(1, W - 1):
        engine.apply_cells(W, W - 1, 1, moduli, dm.data_ptr(), db.data_ptr(), stream)
    torch.cuda.synchronize()
    return dm


@pytest.mark.parametrize("lanes", [1, 4, 8, 14, 16])
def test_noalloc_every_panel_layout(engine, lanes):
    # 1, 4 and 8 lanes are one panel; 14 is panels {0-7}, {8-11}, {12-13}; 16 is
    # the fixed scratch's limit, two 8-wide panels.
    import torch
    n = 9
    moduli = orc.largest_primes_below_2_32(lanes)
    dm = _final_state(engine, n, moduli)
    want = engine.residues(n, moduli, lanes=lanes).residues
    for _call in range(2):
        out = torch.full((lanes,), -1, dtype=torch.int32, device="cuda")
        assert noalloc(n + 1, moduli, dm.data_ptr(), out.data_ptr()) == fdp.FDP_OK
        torch.cuda.synchronize()
        assert [int(x) for x in out.cpu().numpy().view(np.uint32)] == want


def test_noalloc_on_a_caller_stream(engine):
    # The caller's own (non-default) stream orders the state, the read-out and
    # the copy back; two calls in a row on it.
    import torch
    n, lanes = 10, 14
    moduli = orc.largest_primes_below_2_32(lanes)
    s = torch.cuda.Stream()
    dm = _final_state(engine, n, moduli, stream=s.cuda_stream)
    want = engine.residues(n, moduli, lanes=lanes).residues
    for _call in range(2):
        with torch.cuda.stream(s):
            out = torch.full((lanes,), -1, dtype=torch.int32, device="cuda")
        assert noalloc(n + 1, moduli, dm.data_ptr(), out.data_ptr(), s.cuda_stream) == fdp.FDP_OK
        s.synchronize()
        assert [int(x) for x in out.cpu().numpy().view(np.uint32)] == want


def test_noalloc_rejects_sizes_beyond_its_fixed_scratch():
    import torch
    dummy = torch.zeros(64, dtype=torch.int32, device="cuda")
    assert noalloc(13, [7] * 17, dummy.data_ptr(), dummy.data_ptr()) == fdp.FDP_ERR_ARGS
    assert b"16" in fdp.lib().fdp_last_error()
    assert noalloc(29, [7], dummy.data_ptr(), dummy.data_ptr()) == fdp.FDP_ERR_ARGS
    assert noalloc(13, [1], dummy.data_ptr(), dummy.data_ptr()) == fdp.FDP_ERR_MODULUS
