#!/usr/bin/env python3
"""Regenerate tests/golden/path_bound.json from the reference's own
scripts/solve/path_bound.py (needs the reference tree; run from the repo root):

    python tests/golden/gen_path_bound.py <reference tree>
"""
import json
import os
import sys

if len(sys.argv) != 2 or not os.path.isfile(os.path.join(sys.argv[1], "scripts", "solve", "path_bound.py")):
    sys.exit("usage: gen_path_bound.py <reference tree containing scripts/solve/path_bound.py>")
ref = sys.argv[1]
sys.path.insert(0, os.path.join(ref, "scripts", "solve"))
import path_bound  # noqa: E402

out = {"primes": path_bound.PRIMES, "bounds": {}}
for n in range(1, 28):
    bound, parts = path_bound.simple_path_upper_bound(n)
    primes = path_bound.primes_for_bound(bound) if n >= 2 else [path_bound.PRIMES[0]]
    out["bounds"][str(n)] = {"bound": str(bound), "bits": bound.bit_length(), "strips": parts,
                             "crt_primes": len(primes)}
here = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(here, "path_bound.json"), "w") as f:
    json.dump(out, f, indent=1, sort_keys=True)
    f.write("\n")
print("wrote path_bound.json")
