"""Every entry point that runs residue passes reports a kernel's give-up on a
bounded wait as a failure, not as residues.

The failure is planted on the host (fdp_test_inject_pass_errors sets the
computation's device error word before its passes run, exactly what a kernel
that gives up writes), so no kernel is made to fail.  Each computation owns its
word: a planted failure in one request leaves the others' results intact."""
import pytest

import fdp
import oracle_lib as orc

pytestmark = pytest.mark.gpu

MODS = [4294967291, 4294966997]


def test_run_sync_reports_a_planted_failure(engine):
    fdp.inject_pass_errors(1)
    with pytest.raises(fdp.FdpError) as e:
        engine.residues(9, MODS, lanes=2)
    assert e.value.status == fdp.FDP_ERR_CUDA and "bounded wait" in str(e.value)
    assert engine.residues(9, MODS, lanes=2).residues == [2674633373, 3332982389]


def test_run_multi_sync_reports_a_planted_failure(engine):
    fdp.inject_pass_errors(1)
    with pytest.raises(fdp.FdpError) as e:
        engine.residues_multi([(9, MODS), (8, MODS)])
    assert e.value.status == fdp.FDP_ERR_CUDA and "problem 0" in str(e.value)
    got, _ = engine.residues_multi([(9, MODS), (8, MODS)])
    assert got == [[2674633373, 3332982389], [orc.residue(8, m) for m in MODS]]


def test_server_fails_only_the_request_that_failed(engine):
    engine.server_start(1 << 30, max_active=4, max_lanes=2)
    try:
        fdp.inject_pass_errors(1)
        bad = engine.submit(9, MODS)
        with pytest.raises(fdp.FdpError) as e:
            engine.wait(bad, timeout_ms=120000)
        assert e.value.status == fdp.FDP_ERR_CUDA and "bounded wait" in str(e.value)
        good = engine.submit(9, MODS)
        assert engine.wait(good, timeout_ms=120000)["residues"] == [2674633373, 3332982389]
        st = engine.server_stats()
        assert st["failed"] == 1 and st["completed"] == 1
    finally:
        fdp.inject_pass_errors(0)
        engine.server_stop()
