"""Operator surface on the device: canonical rank / unrank and the ternary
rank index, against the oracle and the definition."""
import numpy as np
import pytest

import oracle_lib as orc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("width", [1, 2, 5, 9, 13, 23, 28])
def test_rank_unrank_roundtrip(engine, width):
    import torch
    M = orc.main_states(width)
    rng = np.random.default_rng(width)
    ranks = np.unique(np.concatenate([rng.integers(0, M, size=min(M, 4096), dtype=np.uint64),
                                      np.array([0, M - 1], dtype=np.uint64)]))
    dr = torch.from_numpy(ranks.view(np.int64)).cuda()
    dw = torch.empty_like(dr)
    back = torch.empty_like(dr)
    engine.unrank_words(width, dr.data_ptr(), dw.data_ptr(), len(ranks))
    engine.rank_words(width, dw.data_ptr(), back.data_ptr(), len(ranks))
    torch.cuda.synchronize()
    words = dw.cpu().numpy().view(np.uint64)
    assert np.array_equal(back.cpu().numpy().view(np.uint64), ranks)
    for r, w in list(zip(ranks, words))[:256]:
        assert orc.unrank(int(r), width) == int(w)


def _ternary_words(max_width):
    """Every code of widths 0..max_width with its rank: digit p of the rank in
    base 3 is the two-bit symbol at position p."""
    codes, want = [], []
    for width in range(0, max_width + 1):
        ranks = np.arange(3 ** width, dtype=np.uint64)
        code = np.zeros_like(ranks)
        n = ranks.copy()
        for p in range(width):
            code |= (n % 3) << np.uint64(2 * p)
            n //= 3
        codes.append(code)
        want.append(ranks)
    return np.concatenate(codes).astype(np.uint32), np.concatenate(want).astype(np.uint32)


def test_ternary_index(engine):
    # tests/ternary_rank_index_test.cpp:7-27: a bijection onto [0, 3^width) for
    # widths 0..14, by the scalar conversion and by 4- and 7-symbol chunks.
    import torch
    codes, want = _ternary_words(14)
    c = torch.from_numpy(codes.view(np.int32)).cuda()
    for chunk in (None, 4, 7):
        out = torch.full_like(c, -1)
        if chunk is None:
            engine.ternary_index(c.data_ptr(), out.data_ptr(), len(codes))
        else:
            engine.ternary_index_chunked(chunk, c.data_ptr(), out.data_ptr(), len(codes))
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want), chunk


def test_ternary_index_chunk_must_be_4_or_7(engine):
    import fdp
    import torch
    c = torch.zeros(4, dtype=torch.int32, device="cuda")
    with pytest.raises(fdp.FdpError):
        engine.ternary_index_chunked(5, c.data_ptr(), c.data_ptr(), 4)
