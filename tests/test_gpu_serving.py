"""Serving loop: continuous batching under an HBM budget.  Every request's
residues must be the same in the mix as alone (fdp_run_sync), admission must
respect the budget and the slot count, and every wait is bounded."""
import random

import pytest

import fdp
import oracle_lib as orc

pytestmark = pytest.mark.gpu

P = orc.largest_primes_below_2_32(48)


@pytest.fixture(scope="module")
def server_engine():
    eng = fdp.Engine(0)
    yield eng
    eng.close()


def test_results_in_the_mix_equal_results_alone(server_engine):
    eng = server_engine
    rng = random.Random(0)
    reqs = []
    for _ in range(40):
        n = rng.randint(6, 16)
        k = rng.randint(1, 8)
        reqs.append((n, P[:k] if rng.random() < 0.5 else rng.sample(P, k)))
    eng.server_start(hbm_budget_bytes=8 << 30, max_active=8, max_lanes=4)
    try:
        ids = [eng.submit(n, mods) for n, mods in reqs]
        results = [eng.wait(rid, timeout_ms=120000) for rid in ids]
        stats = eng.server_stats()
    finally:
        eng.server_stop()
    assert stats["completed"] == 40 and stats["failed"] == 0
    assert stats["peak_running"] > 1  # requests overlapped on the device
    assert stats["peak_bytes_in_use"] <= 8 << 30
    for (n, mods), res in zip(reqs, results):
        assert res is not None
        alone = eng.residues(n, mods, lanes=min(len(mods), 16)).residues
        assert res["residues"] == alone, (n, mods)
        if n <= 10:
            assert res["residues"] == [orc.residue(n, m) for m in mods]
        assert res["passes"] == (len(mods) + 3) // 4 and res["latency_s"] >= res["run_s"]


def test_same_n_requests_share_passes(server_engine):
    # Requests of one n whose moduli fit one pass together ride in the same
    # lanes: fewer passes than requests, and every result equal to it alone.
    eng = server_engine
    rng = random.Random(3)
    reqs = [(13 if i % 2 else 14, rng.sample(P, rng.randint(1, 3))) for i in range(24)]
    eng.server_start(hbm_budget_bytes=4 << 30, max_active=1, max_lanes=8)
    try:
        ids = [eng.submit(n, mods) for n, mods in reqs]
        results = [eng.wait(rid, timeout_ms=120000) for rid in ids]
        stats = eng.server_stats()
    finally:
        eng.server_stop()
    assert stats["completed"] == 24 and stats["failed"] == 0
    assert any(r["lanes"] > len(mods) for (_, mods), r in zip(reqs, results))  # some rode in another's lanes
    assert all(r["lanes"] <= 8 and r["passes"] == 1 for r in results)
    for (n, mods), res in zip(reqs, results):
        assert res["residues"] == eng.residues(n, mods, lanes=len(mods)).residues, (n, mods)


def test_budget_limits_admission(server_engine):
    eng = server_engine
    need = fdp.plan(17, P[:4], lanes=4).state_bytes
    eng.server_start(hbm_budget_bytes=int(need * 2.5), max_active=8, max_lanes=4)
    try:
        ids = [eng.submit(17, P[i:i + 4]) for i in range(6)]
        res = [eng.wait(rid, timeout_ms=120000) for rid in ids]
        stats = eng.server_stats()
    finally:
        eng.server_stop()
    assert stats["peak_running"] <= 2 and stats["completed"] == 6
    assert stats["peak_bytes_in_use"] <= int(need * 2.5)
    want = eng.residues(17, P[:9], lanes=9).residues
    for i, r in enumerate(res):
        assert r["residues"] == want[i:i + 4]
    assert max(r["queue_s"] for r in res) > 0


def test_rejects_request_larger_than_budget(server_engine):
    eng = server_engine
    eng.server_start(hbm_budget_bytes=1 << 30, max_active=2, max_lanes=8)
    try:
        with pytest.raises(fdp.FdpError) as e:
            eng.submit(22, P[:8])
        assert e.value.status == fdp.FDP_ERR_HBM
    finally:
        eng.server_stop()


def test_bounded_wait_and_stop(server_engine):
    eng = server_engine
    eng.server_start(hbm_budget_bytes=40 << 30, max_active=1, max_lanes=4)
    try:
        first = eng.submit(20, P[:4])
        queued = eng.submit(20, P[4:8])
        assert eng.wait(first, timeout_ms=1) is None  # runs for ~1 s: the 1 ms wait times out
        assert eng.poll(queued) is None
        r = eng.wait(first, timeout_ms=120000)
        assert r["residues"][0] == 2308006916  # scripts/test/groupbatch-scratch.py:17
        late = eng.submit(20, P[8:12])
    finally:
        eng.server_stop()
    # stop: the running or queued request either finished or failed cleanly
    with pytest.raises(fdp.FdpError):
        eng.poll(late)
