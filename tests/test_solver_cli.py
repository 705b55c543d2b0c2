"""The oneesan_solver process contract (argv positions, stdout tokens, exit
codes), checked like tests/test_solver_contract.py and scripts/solve/solver_output.py
of the reference."""
import math
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SOLVER = os.path.join(ROOT, "oneesan-gpu_b200", "oneesan_solver")

_UINT = re.compile(r"(?:0|[1-9][0-9]*)\Z")
_FLOAT = re.compile(r"(?:0|[1-9][0-9]*)(?:\.[0-9]+)?(?:[eE][+-]?[0-9]+)?\Z")


def parse_result_line(line):
    """Strict parse with the rules of scripts/solve/solver_output.py:25-74."""
    keys = ("n", "residue", "modulus", "wall_s")
    vals = {}
    for tok in line.split():
        for k in keys:
            if tok.startswith(k + "="):
                assert k not in vals, f"duplicate {k}"
                vals[k] = tok[len(k) + 1:]
    if not any(k in vals for k in ("residue", "modulus", "wall_s")):
        return None
    assert all(k in vals for k in keys)
    for k in ("n", "residue", "modulus"):
        assert _UINT.fullmatch(vals[k]), vals[k]
    assert _FLOAT.fullmatch(vals["wall_s"]) and math.isfinite(float(vals["wall_s"]))
    return int(vals["n"]), int(vals["residue"]), int(vals["modulus"]), float(vals["wall_s"])


def run(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([SOLVER, *map(str, args)], capture_output=True, text=True, env=e, timeout=600)


pytestmark = pytest.mark.skipif(not os.path.exists(SOLVER), reason="oneesan_solver not built")


def test_plan_only_needs_no_gpu():
    r = run(22, 512, 14, 1, 4294967291, 4294967279, env={"GRIDFP_PLAN_ONLY": "1"})
    assert r.returncode == 0
    plan = dict(re.findall(r"(\w+)=(\S+)", r.stderr.splitlines()[0]))
    assert plan["main"] == "2062967382" and plan["blocked"] == "728997192"
    assert plan["scratch_fits"] == "1" and "PLAN crt_moduli=2" in r.stderr


def test_rejects_bad_modulus():
    assert run(9, 1, 14, 1, 1).returncode == 1
    assert run(9, 1, 14, 1, 4294967296).returncode == 1
    assert run(9, 1, 14, 1, "12x").returncode == 1


def test_rejects_bad_n():
    assert run(0, 1, 14, 1, 7).returncode == 1
    assert run(28, 1, 14, 1, 7).returncode == 1


@pytest.mark.gpu
def test_result_lines_in_argument_order():
    mods = [4294967291, 4294966997, 2147483647]
    r = run(9, 512, 14, 1, *mods)
    assert r.returncode == 0, r.stderr
    rows = [parse_result_line(l) for l in r.stdout.splitlines()]
    rows = [x for x in rows if x]
    assert [x[2] for x in rows] == mods and all(x[0] == 9 for x in rows)
    assert rows[0][1] == 2674633373 and rows[1][1] == 3332982389
    line = r.stdout.splitlines()[0]
    pos = [line.index(t) for t in (" n=", "residue=", "modulus=", "wall_s=")]
    assert pos == sorted(pos)


@pytest.mark.gpu
def test_plain_lanes_env():
    r = run(12, 512, 14, 1, 4294967291, 4294966997, env={"FDP_LANES": "1"})
    b = run(12, 512, 14, 1, 4294967291, 4294966997)
    assert r.returncode == 0 and b.returncode == 0
    res = lambda out: [parse_result_line(l)[1] for l in out.splitlines() if parse_result_line(l)]
    assert res(r.stdout) == res(b.stdout)
