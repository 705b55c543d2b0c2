"""The multi-GPU path of bench.py on the CPU: world_size 2 over gloo.

bench.py --gpus N runs N independent replicas (residues are independent, so
the path has no data-path collective); the process group only lines the ranks
up around the timed region and takes the max over ranks of the times.  These
tests drive the same Replicas class with the gloo backend and host tensors:
the whole-job throughput must use the slowest rank, every rank must agree on
it, and the reference arm must run on rank 0 only."""
import json
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(body: str, world: int = 2, timeout: float = 120.0):
    port = _free_port()
    script = textwrap.dedent(f"""
        import json, os, sys
        sys.path.insert(0, {ROOT!r})
        import bench
        {textwrap.indent(textwrap.dedent(body), '        ').strip()}
    """)
    procs = []
    for r in range(world):
        env = dict(os.environ, WORLD_SIZE=str(world), RANK=str(r), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", script], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            o, e = p.communicate()
        assert p.returncode == 0, e
        outs.append(o)
    return outs


def test_throughput_uses_the_slowest_rank_on_every_rank():
    outs = _run_ranks("""
        g = bench.Replicas("gloo", timeout_s=60)
        g.barrier()
        seconds = 10.0 if g.rank == 0 else 25.0   # rank 1 is the slower replica
        value = g.throughput(14, seconds)
        print(json.dumps({"rank": g.rank, "world": g.world, "value": value, "max": g.max(seconds)}))
        g.close()
    """)
    got = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    want = 2 * 3600.0 * 14 / 25.0
    for r in got:
        assert r["world"] == 2
        assert abs(r["value"] - want) < 1e-9
        assert r["max"] == 25.0


def test_single_process_needs_no_process_group():
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        env.pop(k, None)
    code = ("import sys; sys.path.insert(0, %r); import bench; g = bench.Replicas('gloo'); "
            "print(g.world, g.throughput(3, 2.0)); g.close()" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.split() == ["1", str(3600.0 * 3 / 2.0)]


def test_reference_arm_runs_on_rank_zero_only():
    # Rank 1 returns at once without work (and prints nothing); rank 0 would
    # time the CPU counter, so only the non-zero rank is exercised here.
    outs = _run_ranks("""
        import types
        if int(os.environ["RANK"]) == 1:
            bench.run_reference(types.SimpleNamespace(warmup=1, steps=1, n=22, k=14, gpus=2))
            print("rank1-done")
        else:
            print("rank0-skipped")
    """)
    assert outs[1].strip() == "rank1-done"
