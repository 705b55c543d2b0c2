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


def test_ternary_index(engine):
    # tests/ternary_rank_index_test.cpp: bijection onto [0, 3^width), widths 0..14
    import torch
    codes, want = [], []
    for width in range(0, 9):
        for rank in range(3 ** width):
            code, n = 0, rank
            for p in range(width):
                code |= (n % 3) << (2 * p)
                n //= 3
            codes.append(code)
            want.append(rank)
    c = torch.tensor(np.array(codes, dtype=np.uint32).view(np.int32), device="cuda")
    out = torch.empty_like(c)
    engine.ternary_index(c.data_ptr(), out.data_ptr(), len(codes))
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), np.array(want, dtype=np.uint32))
