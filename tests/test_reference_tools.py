"""The solver's output read by the reference's own Python tools, imported from
the reference tree (skipped where it is absent):

* scripts/run/autotune.py:189-200 -- the tuner's planning half: `fields`
  parses the `PLAN n=` line of GRIDFP_PLAN_ONLY=1 and `fits` admits a
  configuration from scratch_fits, dp_peak_gib and row6_peak_gib;
* scripts/solve/solver_output.py:25-74 -- the strict result-line parser the
  exact runner uses, applied to result lines this solver printed on a B200
  (tests/golden/solver_stdout_n9.txt, the stdout of
  `oneesan-gpu_b200/oneesan_solver 9 512 14 1 4294967291 4294966997 2147483647`)."""
import importlib.util
import os
import subprocess
import sys
from types import SimpleNamespace

import pytest

import oracle_lib as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SOLVER = os.path.join(ROOT, "oneesan-gpu_b200", "oneesan_solver")
SOLVER_LINES = os.path.join(ROOT, "tests", "golden", "solver_stdout_n9.txt")
REF = orc.reference_root()

pytestmark = pytest.mark.skipif(REF is None, reason="reference tree not available")

GIB = 1 << 30
B200_FREE = 183359 * (1 << 20)  # nvidia-smi's memory.total of a B200


def _load(rel, name):
    spec = importlib.util.spec_from_file_location(name, os.path.join(REF, rel))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod  # dataclasses look their module up while it executes
    spec.loader.exec_module(mod)
    return mod


def _plan_text(n, moduli, gpus=1):
    env = dict(os.environ, GRIDFP_PLAN_ONLY="1")
    r = subprocess.run([SOLVER, str(n), "16384", "14", str(gpus), *map(str, moduli)], capture_output=True,
                       text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    return r.stdout + r.stderr  # the tuner logs both streams into one file


@pytest.mark.skipif(not os.path.exists(SOLVER), reason="oneesan_solver not built")
@pytest.mark.parametrize("n,k,admitted", [(20, 4, True), (22, 14, True), (23, 5, True), (23, 7, False)])
def test_plan_line_read_by_reference_autotuner(n, k, admitted):
    tune = _load("scripts/run/autotune.py", "reference_autotune")
    rows = tune.fields(_plan_text(n, orc.largest_primes_below_2_32(k)), "PLAN n=")
    assert len(rows) == 1 and int(rows[0]["n"]) == n and int(rows[0]["gpus"]) == 1
    plan = rows[0]
    config = SimpleNamespace(devices=(0,))
    hardware = {"gpus": [{"free_bytes": B200_FREE}]}
    assert tune.fits(plan, config, hardware, 1024) is admitted
    # The peaks cover the whole resident state of the pass.
    state_gib = 4 * (int(plan["main"]) + int(plan["blocked"])) * int(plan["lanes"]) / GIB
    assert float(plan["dp_peak_gib"]) >= state_gib and float(plan["row6_peak_gib"]) >= state_gib


@pytest.mark.skipif(not os.path.exists(SOLVER), reason="oneesan_solver not built")
def test_multi_gpu_plan_is_not_admitted():
    tune = _load("scripts/run/autotune.py", "reference_autotune")
    rows = tune.fields(_plan_text(20, [4294967291], gpus=2), "PLAN n=")
    assert len(rows) == 1 and int(rows[0]["gpus"]) == 2 and rows[0]["scratch_fits"] == "0"
    config = SimpleNamespace(devices=(0, 1))
    hardware = {"gpus": [{"free_bytes": B200_FREE}] * 2}
    assert tune.fits(rows[0], config, hardware, 1024) is False


def test_solver_result_lines_parse_with_reference_parser():
    if not os.path.exists(SOLVER_LINES):
        pytest.skip("no captured solver output")
    parse = _load("scripts/solve/solver_output.py", "reference_solver_output").parse_result_line
    with open(SOLVER_LINES) as f:
        rows = [parse(line) for line in f]
    rows = [r for r in rows if r is not None]
    mods = [4294967291, 4294966997, 2147483647]
    assert [r.modulus for r in rows] == mods and all(r.n == 9 for r in rows)
    assert [r.residue for r in rows] == [orc.residue(9, m) for m in mods]
    assert rows[0].residue == 2674633373 and rows[1].residue == 3332982389  # scripts/test/groupbatch-runtime.py:17
