"""The benchmark configurations on the GPU, each residue pinned to the
reference's own CPU path or to a value the reference publishes.

* n = 18 and n = 20, the four largest primes below 2^32, plain (one modulus
  per pass) and batched (four per pass): equal to the reference's CPU counter
  (third_party/ggcount, tests/golden/ggcount_residues.json, made by
  tests/golden/gen_ggcount_residues.py);
* n = 21: equal to the same counter for two moduli;
* n = 22 exact count: the 14 CRT residues in one batched pass of the C++
  driver, every drop-one CRT subset reconstructing the same integer, and the
  residue mod 4294967291 equal to the published 1245069298
  (docs/results/groupbatch-interleaved-2026-09-05.json:1027 of the reference);
* n = 23, one modulus: the published residue 2762394459 mod 4294967291
  (docs/b300-hbm32.md:382-385 of the reference).
"""
import json
import os
import re
import subprocess

import pytest

import fdp
import oracle_lib as orc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXACT = os.path.join(ROOT, "oneesan-gpu_b200", "oneesan_exact")
with open(os.path.join(ROOT, "tests", "golden", "ggcount_residues.json")) as _f:
    GGCOUNT = json.load(_f)["residues"]
TOP4 = orc.largest_primes_below_2_32(4)


def ggcount(n):
    """{modulus: residue} the reference's CPU counter gave at grid size n."""
    return {e["modulus"]: e["residue"] for e in GGCOUNT if e["n"] == n}


@pytest.mark.parametrize("n", [18, 20])
def test_four_largest_primes_plain_and_batched_match_ggcount(engine, n):
    want = ggcount(n)
    assert set(TOP4) <= set(want), f"fixture lacks n={n} residues for {TOP4}"
    want = [want[m] for m in TOP4]
    assert engine.residues(n, TOP4, lanes=1).residues == want
    assert engine.residues(n, TOP4, lanes=4).residues == want


def test_n21_matches_ggcount(engine):
    want = ggcount(21)
    mods = [4294967291, 4294966997]
    assert set(mods) <= set(want), "fixture lacks the n=21 residues"
    assert engine.residues(21, mods, lanes=2).residues == [want[m] for m in mods]


def test_n22_exact_count_with_drop_one_cross_check(tmp_path):
    # Config 3: the 14 CRT primes the path bound needs, one batched pass.
    work = tmp_path / "n22"
    r = subprocess.run([EXACT, "22", "--work-dir", str(work), "--lanes", "14"], capture_output=True, text=True,
                       timeout=1200)
    assert r.returncode == 0, r.stderr
    m = re.search(r"crt cross-check: (\d+) of (\d+) drop-one subsets", r.stderr)
    assert m and m.group(1) == m.group(2) == "14", r.stderr
    assert "primes_used=14" in r.stdout
    ck = json.loads((work / "checkpoint.json").read_text())
    assert ck["residues"]["4294967291"]["residue"] == 1245069298
    man = json.loads((work / "exact_manifest.json").read_text())
    assert man["primes_used"] == 14 and int(man["exact_decimal"]) > 0


def test_n23_published_residue():
    # Config 5 at one modulus: 29.5 GiB of state, 64-bit indices.  A context of
    # its own, released at the end, so the state does not stay resident.
    with fdp.Engine(0) as eng:
        assert eng.residues(23, [4294967291], lanes=1).residues == [2762394459]
