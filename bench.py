#!/usr/bin/env python3
"""Benchmark of the frontier-DP hot path on B200.

Workload (default): n = 22 exact count, the 14 largest primes below 2^32 (the
CRT prime count the checkerboard-strip bound needs at n = 22), all 14 residues
in one batched pass (lanes = 14, one CUDA graph).  A step is one such pass:
row-0 initialiser, 21 row sweeps of 22 cells over the HBM-resident state
(145.6 GiB, far above L2, so no flush is needed), first-row dot product.

value    residues/hour from the device time of the captured pass (CUDA events
         on the engine's stream), max over ranks.
e2e      residues/hour through the public C ABI call fdp_run_sync from host
         buffers (moduli in, residues out) including graph capture.
roofline the per-cell transition kernel: algorithmic bytes per cell
         (fdp_cell_bytes: 4 x words that must be read + 4 x words that can
         change, per modulus) over the cell's CUDA-event duration (with 14
         lanes a cell is two launches, one per lane span of at most 8).

--impl reference times the reference's own CPU counter (third_party/ggcount,
built unmodified into oracle/_ref) on all host threads: each step is one
n = 18 residue (the plain configuration the reference's CPU path runs), scaled
to residues/hour at n = 22 by the ratio of frontier transitions per residue
(stated in the line).  Measured here, that ratio favours the CPU counter: its
n = 20 residue takes 12.4x its n = 18 residue, where transitions grow 9.8x.
That arm loads nothing of this repository's engine.

Multi-GPU: replicas only (moduli are independent; no data-path collective).
Each rank runs the same workload; value is the sum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "oneesan-gpu_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "residues/hour and frontier transitions/s at n=22 on 1 B200 (batched vs plain), HBM GB/s"


def primes_below_2_32(count: int) -> list[int]:
    def is_prime(x: int) -> bool:
        for q in (2, 3, 5, 7, 11, 13):
            if x % q == 0:
                return x == q
        d, s = x - 1, 0
        while d % 2 == 0:
            d //= 2
            s += 1
        for a in (2, 3, 5, 7, 11, 13, 17):
            y = pow(a, d, x)
            if y in (1, x - 1):
                continue
            for _ in range(s - 1):
                y = y * y % x
                if y == x - 1:
                    break
            else:
                return False
        return True
    out, x = [], (1 << 32) - 1
    while len(out) < count:
        if is_prime(x):
            out.append(x)
        x -= 1
    return out


def measured_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


# Residues the reference publishes for its GPU solvers (n, modulus) -> residue.
PUBLISHED = {
    (22, 4294967291): 1245069298,  # docs/results/groupbatch-interleaved-2026-09-05.json:1027
    (21, 4294967291): 998035516,   # docs/b300-hbm32.md:554
    (21, 4294966997): 2124618149,  # scripts/run/autotune.py:28
    (20, 4294967291): 2308006916,  # scripts/test/groupbatch-scratch.py:17
    (20, 4294966997): 3704549185,
    (18, 4294967291): 503411004,   # docs/results/reverse-algorithm-2026-09-05.md:53
    (23, 4294967291): 2762394459,  # docs/b300-hbm32.md:382-385
}


def published_check(n: int, moduli, residues) -> dict:
    """Compare the residues with every published value for this n; a mismatch
    ends the run (a wrong count has no throughput)."""
    checked = []
    for m, r in zip(moduli, residues):
        want = PUBLISHED.get((n, m))
        if want is not None:
            if r != want:
                raise SystemExit(f"n={n} mod {m}: residue {r} != published {want}")
            checked.append({"modulus": m, "residue": r})
    return {"published_residues_matched": checked}


def committed_traffic(n: int, lanes: int):
    """DRAM bytes per cell (all of the cell's lane-span launches) of the cell
    kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "cell_kernel_traffic.txt")
    if not os.path.exists(path):
        return None
    pat = re.compile(rf"^n={n}\s+lanes={lanes}\s+dram_bytes_per_cell=(\d+)")
    with open(path) as f:
        for line in f:
            m = pat.match(line.strip())
            if m:
                return int(m.group(1))
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index, self.samples, self.proc, self.thread = index, [], None, None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        def pump():
            for line in self.proc.stdout:
                self.samples.append([x.strip() for x in line.split(",")])
        self.thread = threading.Thread(target=pump, daemon=True)
        self.thread.start()

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[1]))
                mx.append(float(s[2]))
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


CPU_SAMPLE_N = 18          # the plain configuration the reference's CPU path runs
CPU_SAMPLE_MOD = 4294967291
CPU_SAMPLE_RESIDUE = 503411004  # docs/results/reverse-algorithm-2026-09-05.md:53 of the reference


def ggcount_sample(threads: int | None = None):
    """Time the reference's CPU counter on one residue: n = 18 mod 4294967291,
    all host threads (OpenMP)."""
    import oracle_lib as orc
    exe = orc.GGCOUNT
    n_s, mod = CPU_SAMPLE_N, CPU_SAMPLE_MOD
    env = dict(os.environ)
    cores = threads or os.cpu_count() or 1
    env["OMP_NUM_THREADS"] = str(cores)
    if os.path.exists(exe):
        t0 = time.perf_counter()
        out = subprocess.run([exe, "-q", str(n_s), f"%{mod}"], check=True, capture_output=True, text=True,
                             env=env).stdout
        dt = time.perf_counter() - t0
        kind = "reference"
        res = int(out.split()[0])
        if res != CPU_SAMPLE_RESIDUE:
            raise SystemExit(f"ggcount n={n_s} mod {mod} gave {res}, expected {CPU_SAMPLE_RESIDUE}")
    else:  # nothing prebuilt: the oracle port, one thread, a smaller grid
        n_s = 13
        t0 = time.perf_counter()
        res = orc.residue(n_s, mod)
        dt = time.perf_counter() - t0
        kind, cores = "port", 1
    return {"n": n_s, "modulus": mod, "residue": res, "seconds": dt, "kind": kind, "cores": cores,
            "cpu": cpu_model(), "nproc": os.cpu_count()}


def transitions_per_residue(n: int) -> int:
    """Frontier transitions of a full residue (every row swept): (W-2) rows x
    (W-1) cells x (M + D) states, with M, D the canonical state counts (words
    of W and W-1 symbols from height 1 to 0, N keeps the height, R lowers and
    L raises it).  Pure Python: the reference arm loads none of the engine."""
    W = n + 1
    H = [[0] * (W + 3) for _ in range(W + 1)]
    H[0][0] = 1
    for w in range(1, W + 1):
        for h in range(W + 2):
            H[w][h] = H[w - 1][h] + (H[w - 1][h - 1] if h else 0) + H[w - 1][h + 1]
    return (W - 2) * (W - 1) * (H[W][1] + H[W - 1][1])


def cpu_scale(sample: dict, n: int) -> float:
    """Factor from the sample's seconds per residue to size n's, by frontier
    transitions per residue."""
    return transitions_per_residue(n) / transitions_per_residue(sample["n"])


def scale_cpu(sample: dict, n: int) -> float:
    """CPU residues/hour at size n, scaled from the sample by frontier transitions."""
    return 3600.0 / (sample["seconds"] * cpu_scale(sample, n))


def cpu_baseline_record(sample: dict, n: int, value: float) -> dict:
    return {"value": value, "unit": "residues/hour", "cores": sample["cores"], "kind": sample["kind"],
            "cpu": sample["cpu"], "nproc": sample["nproc"],
            "sample": (f"ggcount_multi -q {sample['n']} %{sample['modulus']}: one residue "
                       f"({sample['residue']}) in {sample['seconds']:.2f} s on {sample['cores']} threads, "
                       f"scaled to n={n} by frontier transitions per residue (x{cpu_scale(sample, n):.2f})"),
            "scale_to_n": n, "scale_factor": cpu_scale(sample, n), "sample_seconds": sample["seconds"]}


def bench_config(n: int, k: int, world: int) -> dict:
    """The workload, the same object in both arms' lines."""
    return {"workload": f"n={n} exact count: the {k} largest primes below 2^32 (the CRT primes the "
                        f"checkerboard-strip bound needs)", "n": n, "moduli": k,
            "l2": "state far larger than L2 (126 MB); no flush needed",
            "parallelism": f"replicas x{world}"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    vals, samples = [], []
    for i in range(args.warmup + args.steps):
        s = ggcount_sample()
        if i >= args.warmup:
            vals.append(scale_cpu(s, args.n))
            samples.append(s)
    mean_s = statistics.mean(x["seconds"] for x in samples)
    s0 = dict(samples[-1], seconds=mean_s)
    v = scale_cpu(s0, args.n)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "residues/hour", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * mean_s,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "none: the DP has no input data",
        "config": bench_config(args.n, args.k, world),
        "cpu_baseline": cpu_baseline_record(s0, args.n, v),
        "e2e": {"value": v, "unit": "residues/hour", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "step_seconds": [x["seconds"] for x in samples],
    }
    print(json.dumps(line), flush=True)


class Replicas:
    """One process per GPU, each running the whole workload on its own moduli
    replica (weak scaling): residues are independent, so there is no
    data-path collective.  The process group only lines the ranks up around
    the timed region and takes the max over ranks of the times; the job's
    throughput is world x per-replica work / that max.  backend "nccl" on
    GPUs; "gloo" (host tensors) runs the same logic without a GPU."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 600.0):
        import torch
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend, self.dist = backend, None
        self.device = torch.device("cuda", self.local) if backend == "nccl" else torch.device("cpu")
        if backend == "nccl":
            torch.cuda.set_device(self.local)
        if self.world > 1:
            import torch.distributed as dist
            from datetime import timedelta
            kw = {"device_id": self.device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
            self.dist = dist

    def barrier(self) -> None:
        import torch
        if self.dist is not None:
            self.dist.barrier()
        if self.backend == "nccl":
            torch.cuda.synchronize()

    def max(self, x: float) -> float:
        import torch
        if self.dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, residues_per_replica: int, seconds: float) -> float:
        """Whole-job residues/hour: every replica's residues over the slowest
        replica's time (max over ranks)."""
        return self.world * 3600.0 * residues_per_replica / self.max(seconds)

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def run_ours(args) -> None:
    import fdp

    group = Replicas("nccl")
    world, rank, local = group.world, group.rank, group.local
    barrier = group.barrier
    max_over_ranks = group.max

    n, k = args.n, args.k
    moduli = primes_below_2_32(k)
    W = n + 1
    eng = fdp.Engine(local)
    tuned = None
    if args.lanes:
        lanes = args.lanes
    else:  # the autotuner picks residues per pass, panel strategy and CTA size
        tuned = eng.autotune(n, moduli, max_lanes=min(k, fdp.MAX_LANES), repeats=1)
        lanes = tuned["best"]["lanes"]
    plan = fdp.plan(n, moduli, lanes)

    # Warm-up (graph capture, table upload, first-touch of the state buffers).
    for _ in range(args.warmup):
        eng.residues(n, moduli, lanes)
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    dev_s, wall_s, launches, results = 0.0, 0.0, 0, None
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = eng.residues(n, moduli, lanes)
        dev_s += r.stats.device_s
        launches += int(r.stats.kernel_launches)
        results = r.residues
    barrier()
    wall_s = time.perf_counter() - t0
    clocks = sampler.stop()
    value = group.throughput(k * args.steps, dev_s)
    e2e = group.throughput(k * args.steps, wall_s)
    dev_s = max_over_ranks(dev_s)
    wall_s = max_over_ranks(wall_s)

    # Plain form: one modulus per launch sequence (lanes = 1), one residue.
    extra = {}
    if rank == 0 and not args.no_plain:
        rp = eng.residues(n, moduli[:1], 1)
        if rp.residues[0] != results[0]:
            raise SystemExit(f"plain/batched mismatch: {rp.residues[0]} != {results[0]}")
        extra["plain"] = {"value": 3600.0 / rp.stats.device_s, "unit": "residues/hour",
                          "sample": "one residue, lanes=1", "device_s": rp.stats.device_s}

    # Roofline of the dominant kernel: per-cell CUDA-event times of one row sweep
    # (a cell of more than 8 lanes is one launch per lane span of at most 8).
    cell_ms = eng.time_cells(n, moduli, lanes, rows=args.profile_rows)
    tuning = eng.get_tuning()
    split = lanes > 8 and not tuning["split_panels"] and tuning["split_spans_min_p"] <= 1
    launches_per_cell = len(fdp.lane_spans(lanes)) if split else 1
    tot_bytes = sum(fdp.cell_bytes(W, p) * lanes for p in range(1, W))
    tot_ms = sum(cell_ms[1:])
    achieved = tot_bytes / (tot_ms * 1e-3) / 1e9
    peaks = measured_peaks()
    traffic = committed_traffic(n, lanes)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
            "kernel": "cell_kernel / cell_stream_kernel (per-cell frontier transition)",
            "peak_source": peaks["source"],
            "alg_bytes_per_cell": tot_bytes / (W - 1), "mean_cell_ms": tot_ms / (W - 1),
            "launches_per_cell": launches_per_cell, "row_ms": tot_ms,
            "cell_gbs": [fdp.cell_bytes(W, p) * lanes / (cell_ms[p] * 1e-3) / 1e9 for p in range(1, W)]}
    # The same bytes over the timed passes' device time: in a pass the two lane
    # spans sweep as concurrent launch chains, which the per-cell timing (one
    # span launch after the other) does not see; the row-k fill and the
    # read-out are inside this time and not in the bytes.
    pass_gbs = plan.alg_bytes_per_residue * k * args.steps / dev_s / 1e9
    roof["pass_gbs"] = pass_gbs
    roof["pass_frac"] = pass_gbs / peaks["hbm_gbs"]
    eng.close()  # frees the state before the sub-runs below

    transitions = plan.transitions_per_residue * k * args.steps * world
    line = {
        "metric": METRIC, "value": value, "unit": "residues/hour", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * dev_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "none: the DP has no input data; the state is generated on the device",
        "config": bench_config(n, k, world),
        "plan": {"lanes": lanes, "passes": plan.passes, "state_gib": plan.state_bytes / 2**30,
                 "tuning": tuning, "autotuned": tuned["best"] if tuned else None},
        "transitions_per_s": transitions / dev_s,
        "residues": results,
        "check": published_check(n, moduli, results),
        "e2e": {"value": e2e, "unit": "residues/hour", "h2d_bytes_per_step": 4 * k,
                "d2h_bytes_per_step": 4 * k},
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clocks,
    }
    line.update(extra)
    if rank == 0 and world == 1 and not args.no_n20:
        line["n20"] = run_n20(local)
    if rank == 0 and world == 1 and not args.no_n23:
        line["n23"] = run_n23(local)
    if rank == 0 and world == 1 and not args.no_serve:
        line["serving"] = run_serving_stream(args.seed, args.serve_requests, args.serve_gap, 0.1,
                                             args.serve_budget_gb, args.serve_slots, args.serve_max_lanes)
    if rank == 0 and world == 1 and not args.no_cpu:
        s = ggcount_sample()
        line["cpu_baseline"] = cpu_baseline_record(s, n, scale_cpu(s, n))
    if rank == 0:
        print(json.dumps(line), flush=True)
    group.close()


def run_n20(device: int) -> dict:
    """Config 2: n = 20, the four largest primes below 2^32, plain (one modulus
    per pass, lanes = 1) and batched (one pass of four lanes); every residue is
    checked against the reference's CPU counter (tests/golden/ggcount_residues.json)."""
    import fdp
    mods = primes_below_2_32(4)
    with open(os.path.join(ROOT, "tests", "golden", "ggcount_residues.json")) as f:
        ref = {e["modulus"]: e["residue"] for e in json.load(f)["residues"] if e["n"] == 20}
    out = {}
    with fdp.Engine(device) as eng:
        for name, lanes in (("plain", 1), ("batched", 4)):
            eng.residues(20, mods, lanes)  # warm-up: tables, capture, first touch
            r = eng.residues(20, mods, lanes)
            if [ref.get(m) for m in mods] != r.residues:
                raise SystemExit(f"n=20 {name}: residues {r.residues} != ggcount {[ref.get(m) for m in mods]}")
            out[name] = {"residues_per_hour": 3600.0 * len(mods) / r.stats.device_s, "device_s": r.stats.device_s,
                         "lanes": lanes}
    out["residues"] = [ref[m] for m in mods]
    out["checked_against"] = "reference CPU counter (ggcount), tests/golden/ggcount_residues.json"
    out["batched_over_plain"] = out["batched"]["residues_per_hour"] / out["plain"]["residues_per_hour"]
    return out


def run_n23(device: int, budget: int = 170 * 10**9) -> dict:
    """Config 5: n = 23 at HBM capacity.  The largest number of the largest
    primes below 2^32 whose state and tables fit the budget runs as one pass;
    its residue mod 4294967291 is checked against the published value."""
    import fdp
    lanes = 0
    for cand in range(fdp.MAX_LANES, 0, -1):
        pl = fdp.plan(23, primes_below_2_32(cand), cand, budget)
        if pl.fits and pl.passes == 1:
            lanes = cand
            break
    if not lanes:
        return {"skipped": "no lane count of n = 23 fits the budget"}
    mods = primes_below_2_32(lanes)
    pl = fdp.plan(23, mods, lanes, budget)
    with fdp.Engine(device) as eng:
        r = eng.residues(23, mods, lanes)
    if r.residues[0] != PUBLISHED[(23, 4294967291)]:
        raise SystemExit(f"n=23 mod 4294967291: residue {r.residues[0]} != published {PUBLISHED[(23, 4294967291)]}")
    return {"lanes": lanes, "budget_gb": budget / 1e9, "state_gib": pl.state_bytes / 2**30,
            "device_s": r.stats.device_s, "residues_per_hour": 3600.0 * lanes / r.stats.device_s,
            "residues": r.residues, "checked": {"modulus": 4294967291, "residue": r.residues[0],
                                                "published": "docs/b300-hbm32.md:382-385 of the reference"}}


def run_serving_stream(seed: int, count: int, gap: float, time_scale: float, budget_gb: float,
                       slots: int, max_lanes: int = 16) -> dict:
    """The serving stream: seeded Poisson arrivals, n ~ U{12..21}, k ~ U{1..8}
    largest-below-2^32 primes, admission under an HBM budget.  Every residue
    is checked against the same request run alone through fdp_run_sync."""
    import random
    import threading as th
    import fdp
    rng = random.Random(seed)
    primes = primes_below_2_32(8)
    reqs, t = [], 0.0
    for _ in range(count):
        t += rng.expovariate(1.0 / gap)
        n = rng.randint(12, 21)
        k = rng.randint(1, 8)
        reqs.append((t * time_scale, n, primes[:k]))
    eng = fdp.Engine(0)
    # Warm-up (tables and kernels for every n of the stream), which also gives
    # every request's residues alone: one run of each n with all 8 primes.
    alone = {}
    for n in sorted({r[1] for r in reqs}):
        alone[n] = eng.residues(n, primes, 8).residues
    eng.close()
    eng = fdp.Engine(0)
    eng.server_start(int(budget_gb * 1e9), max_active=slots, max_lanes=max_lanes)
    ids = [None] * len(reqs)
    t0 = time.perf_counter()

    def submitter():
        for i, (at, n, mods) in enumerate(reqs):
            d = at - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            ids[i] = eng.submit(n, mods)
    sub = th.Thread(target=submitter)
    sub.start()
    sampler = ClockSampler(0)
    sampler.start()
    results = []
    for i in range(len(reqs)):
        while ids[i] is None:
            time.sleep(0.001)
        results.append(eng.wait(ids[i], timeout_ms=3600 * 1000))
    makespan = time.perf_counter() - t0
    sub.join()
    clocks = sampler.stop()
    stats = eng.server_stats()
    eng.server_stop()
    eng.close()
    mismatches = sum(1 for (_, n, mods), r in zip(reqs, results) if r["residues"] != alone[n][:len(mods)])
    if mismatches:
        raise SystemExit(f"serving: {mismatches} requests differ from the same request run alone")
    lat = sorted(r["latency_s"] for r in results)

    def pct(q):
        return lat[min(len(lat) - 1, int(q * len(lat)))]
    residues = sum(len(m) for _, _, m in reqs)
    return {
        "workload": f"seed {seed}: {len(reqs)} requests, Poisson arrivals mean gap {gap} s x time scale "
                    f"{time_scale}, n~U{{12..21}}, k~U{{1..8}} largest primes below 2^32",
        "budget_gb": budget_gb, "slots": slots, "max_lanes": max_lanes,
        "p50_latency_s": pct(0.5), "p99_latency_s": pct(0.99), "max_latency_s": lat[-1],
        "mean_queue_s": statistics.mean(r["queue_s"] for r in results),
        "throughput_residues_per_hour": 3600.0 * residues / makespan,
        "throughput_requests_per_s": len(reqs) / makespan, "makespan_s": makespan,
        "peak_running": stats["peak_running"], "peak_gb_in_use": stats["peak_bytes_in_use"] / 1e9,
        "completed": stats["completed"], "failed": stats["failed"],
        "results_equal_alone": len(reqs) - mismatches, "clocks": clocks,
    }


def run_serving(args) -> None:
    rec = run_serving_stream(args.seed, args.serve_requests, args.serve_gap, args.serve_time_scale,
                             args.serve_budget_gb, args.serve_slots, args.serve_max_lanes)
    line = {"metric": "serving stream latency and throughput (continuous batching)",
            "value": rec["p50_latency_s"], "unit": "s (p50 latency)", "higher_is_better": False, "n_gpus": 1,
            "dtype": "u32", "config": {"workload": rec["workload"], "budget_gb": rec["budget_gb"],
                                       "slots": rec["slots"], "max_lanes": rec["max_lanes"]}}
    line.update(rec)
    print(json.dumps(line), flush=True)


def run_cells_only(args) -> None:
    """One row sweep (cells p = n..1, one launch each) of lanes moduli on the
    engine's resident state; prints the per-cell CUDA-event times."""
    import fdp
    lanes = args.lanes or min(args.k, fdp.MAX_LANES)
    moduli = primes_below_2_32(lanes)
    W = args.n + 1
    with fdp.Engine(0) as eng:
        ms = eng.time_cells(args.n, moduli, lanes, rows=args.profile_rows)
    gbs = [fdp.cell_bytes(W, p) * lanes / (ms[p] * 1e-3) / 1e9 for p in range(1, W)]
    print(json.dumps({"n": args.n, "lanes": lanes, "cell_ms": ms[1:], "cell_gbs": gbs}), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=22)
    ap.add_argument("--k", type=int, default=14)
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--profile-rows", type=int, default=1)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-n20", action="store_true", help="skip the n=20 plain/batched sub-record")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-stream sub-record")
    ap.add_argument("--no-n23", action="store_true", help="skip the n=23 at-capacity sub-record")
    ap.add_argument("--serve", action="store_true", help="run the serving stream instead")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--serve-gap", type=float, default=2.0)
    ap.add_argument("--serve-time-scale", type=float, default=1.0)
    ap.add_argument("--serve-budget-gb", type=float, default=120.0)
    ap.add_argument("--serve-slots", type=int, default=8)
    ap.add_argument("--serve-max-lanes", type=int, default=16,
                    help="residues per pass of a served request, shared by same-n requests that ride along")
    ap.add_argument("--cells-only", action="store_true",
                    help="profiling case: one row sweep of separately launched cells on a resident state")
    args = ap.parse_args()
    if args.serve:
        run_serving(args)
    elif args.cells_only:
        run_cells_only(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
