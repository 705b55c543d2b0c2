#!/usr/bin/env python3
"""Write tests/golden/ggcount_residues.json: residues computed by the
reference's own CPU counter (third_party/ggcount/src/ggcount.cpp:833-940,
built unmodified by `make -C oracle ref` into oracle/_ref/ggcount_multi).

Each entry is one `ggcount_multi -q <n> %<p>` run (one modulus per process,
all host threads through OpenMP), with its wall time and the thread count.
Run from the repository root; existing entries are kept, so the file grows
one run at a time and an interrupted run loses at most the entry in flight:

    python tests/golden/gen_ggcount_residues.py 18:4 20:4 21:4294967291,4294966997

`N:K` asks for the K largest primes below 2^32 at grid size N; `N:p,q,...`
for the listed moduli.
"""
import json
import os
import re
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
from oracle_lib import GGCOUNT, largest_primes_below_2_32  # noqa: E402

OUT = os.path.join(HERE, "ggcount_residues.json")


def parse_spec(spec):
    n, _, rest = spec.partition(":")
    n = int(n)
    if "," in rest or int(rest) > 64:
        return n, [int(x) for x in rest.split(",") if x]
    return n, largest_primes_below_2_32(int(rest))


def main(argv):
    if not argv:
        print(__doc__)
        return 2
    if not os.path.exists(GGCOUNT):
        print(f"missing {GGCOUNT}: run `make -C oracle ref` with the reference tree present",
              file=sys.stderr)
        return 1
    data = {"source": "third_party/ggcount/src/ggcount.cpp (reference CPU counter), "
                      "oracle/_ref/ggcount_multi -q <n> %<p>",
            "threads": os.cpu_count(), "residues": []}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    have = {(e["n"], e["modulus"]) for e in data["residues"]}
    for spec in argv:
        n, mods = parse_spec(spec)
        for p in mods:
            if (n, p) in have:
                continue
            t0 = time.time()
            out = subprocess.run([GGCOUNT, "-q", str(n), f"%{p}"], check=True,
                                 capture_output=True, text=True).stdout
            wall = time.time() - t0
            m = re.match(r"\s*(\d+) \(mod (\d+)\)", out)
            if not m or int(m.group(2)) != p:
                raise RuntimeError(f"unexpected ggcount output: {out!r}")
            data["residues"].append({"n": n, "modulus": p, "residue": int(m.group(1)),
                                     "wall_s": round(wall, 1), "threads": os.cpu_count()})
            data["residues"].sort(key=lambda e: (e["n"], -e["modulus"]))
            have.add((n, p))
            with open(OUT + ".tmp", "w") as f:
                json.dump(data, f, indent=1)
                f.write("\n")
            os.replace(OUT + ".tmp", OUT)
            print(f"n={n} p={p} residue={m.group(1)} wall={wall:.1f}s", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
