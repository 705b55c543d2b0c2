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
roofline the per-cell transition kernel: algorithmic bytes per launch
         (fdp_cell_bytes: 4 x words that must be read + 4 x words that can
         change, per modulus) over its CUDA-event duration.

--impl reference times the reference's own CPU counter (third_party/ggcount,
built unmodified into oracle/_ref) on a bounded sample and scales it to the
same workload by frontier transitions.

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
    """Per-launch DRAM bytes of the cell kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "cell_kernel_traffic.txt")
    if not os.path.exists(path):
        return None
    pat = re.compile(rf"^n={n}\s+lanes={lanes}\s+dram_bytes_per_launch=(\d+)")
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


def ggcount_sample(threads: int | None = None):
    """Time the reference's CPU counter on one bounded sample: n=17, one modulus."""
    import oracle_lib as orc
    exe = orc.GGCOUNT
    n_s, mod = 17, 4294967291
    if not os.path.exists(exe):
        try:
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except (OSError, subprocess.CalledProcessError):
            pass
    env = dict(os.environ)
    cores = threads or os.cpu_count() or 1
    env["OMP_NUM_THREADS"] = str(cores)
    t0 = time.perf_counter()
    if os.path.exists(exe):
        out = subprocess.run([exe, "-q", str(n_s), f"%{mod}"], check=True, capture_output=True, text=True,
                             env=env).stdout
        kind = "reference"
        res = int(out.split()[0])
    else:  # reference tree absent and nothing prebuilt: the oracle port, 1 thread
        n_s = 13
        res = orc.residue(n_s, mod)
        kind, cores = "port", 1
    dt = time.perf_counter() - t0
    return {"n": n_s, "modulus": mod, "residue": res, "seconds": dt, "kind": kind, "cores": cores}


def transitions_per_residue(n: int) -> int:
    import fdp
    W = n + 1
    return (W - 2) * (W - 1) * (fdp.main_states(W) + fdp.blocked_states(W))


def scale_cpu(sample: dict, n: int) -> float:
    """CPU residues/hour at size n, scaled from the sample by frontier transitions."""
    rate = transitions_per_residue(sample["n"]) / sample["seconds"]
    return 3600.0 * rate / transitions_per_residue(n)


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    vals, samples = [], []
    for i in range(args.warmup + args.steps):
        s = ggcount_sample()
        if i >= args.warmup:
            vals.append(scale_cpu(s, args.n))
            samples.append(s)
    v = sum(vals) / len(vals)
    s0 = samples[-1]
    sample_txt = (f"ggcount_multi -q {s0['n']} %{s0['modulus']} (one residue, {s0['cores']} threads, "
                  f"{s0['seconds']:.2f} s), scaled to n={args.n} by frontier transitions per residue")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "residues/hour", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * statistics.mean(x["seconds"] for x in samples),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "none: the DP state is generated by the initialiser",
        "config": {"workload": f"n={args.n} exact count, {args.k} largest primes below 2^32", "n": args.n,
                   "moduli": args.k},
        "cpu_baseline": {"value": v, "unit": "residues/hour", "cores": s0["cores"], "kind": s0["kind"],
                         "sample": sample_txt},
        "e2e": {"value": v, "unit": "residues/hour", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
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

    # Roofline of the dominant kernel: per-cell CUDA-event times of one row sweep.
    cell_ms = eng.time_cells(n, moduli, lanes, rows=args.profile_rows)
    tot_bytes = sum(fdp.cell_bytes(W, p) * lanes for p in range(1, W))
    tot_ms = sum(cell_ms[1:])
    achieved = tot_bytes / (tot_ms * 1e-3) / 1e9
    peaks = measured_peaks()
    traffic = committed_traffic(n, lanes)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
            "kernel": "cell_kernel (per-cell frontier transition)", "peak_source": peaks["source"],
            "alg_bytes_per_launch": tot_bytes / (W - 1), "mean_launch_ms": tot_ms / (W - 1)}

    transitions = plan.transitions_per_residue * k * args.steps * world
    line = {
        "metric": METRIC, "value": value, "unit": "residues/hour", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * dev_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "none: the DP state is generated by the row-0 initialiser",
        "config": {"workload": f"n={n} exact count: {k} largest primes below 2^32, {lanes} residues "
                               f"per pass, all passes in one CUDA graph", "n": n, "moduli": k, "lanes": lanes,
                   "passes": plan.passes, "state_gib": plan.state_bytes / 2**30,
                   "tuning": eng.get_tuning(), "autotuned": tuned["best"] if tuned else None,
                   "l2": "state far larger than L2 (126 MB); no flush needed",
                   "parallelism": f"replicas x{world}"},
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
    if rank == 0 and world == 1 and not args.no_cpu:
        s = ggcount_sample()
        v = scale_cpu(s, n)
        line["cpu_baseline"] = {
            "value": v, "unit": "residues/hour", "cores": s["cores"], "kind": s["kind"],
            "sample": f"ggcount_multi -q {s['n']} %{s['modulus']} one residue in {s['seconds']:.2f} s, "
                      f"scaled to n={n} by frontier transitions per residue"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    group.close()


def run_serving(args) -> None:
    """The serving stream: seeded Poisson arrivals, n ~ U{12..21}, k ~ U{1..8}
    largest-below-2^32 primes, admission under an HBM budget."""
    import random
    import threading as th
    import fdp
    rng = random.Random(args.seed)
    primes = primes_below_2_32(8)
    reqs, t = [], 0.0
    for _ in range(args.serve_requests):
        t += rng.expovariate(1.0 / args.serve_gap)
        n = rng.randint(12, 21)
        k = rng.randint(1, 8)
        reqs.append((t * args.serve_time_scale, n, primes[:k]))
    eng = fdp.Engine(0)
    # warm-up: tables and kernels for every n of the stream
    for n in sorted({r[1] for r in reqs}):
        eng.residues(n, primes[:1], 1)
    eng.server_start(int(args.serve_budget_gb * 1e9), max_active=args.serve_slots, max_lanes=8)
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
        r = eng.wait(ids[i], timeout_ms=3600 * 1000)
        results.append(r)
    makespan = time.perf_counter() - t0
    sub.join()
    clocks = sampler.stop()
    stats = eng.server_stats()
    eng.server_stop()
    lat = sorted(r["latency_s"] for r in results)
    def pct(q):
        return lat[min(len(lat) - 1, int(q * len(lat)))]
    residues = sum(len(m) for _, _, m in reqs)
    line = {
        "metric": "serving stream latency and throughput (continuous batching)", "value": pct(0.5),
        "unit": "s (p50 latency)", "higher_is_better": False, "n_gpus": 1, "dtype": "u32",
        "config": {"workload": f"seed {args.seed}: {len(reqs)} requests, Poisson arrivals mean gap "
                               f"{args.serve_gap} s x time scale {args.serve_time_scale}, n~U{{12..21}}, "
                               f"k~U{{1..8}} largest primes below 2^32", "budget_gb": args.serve_budget_gb,
                   "slots": args.serve_slots, "max_lanes": 8},
        "p50_latency_s": pct(0.5), "p99_latency_s": pct(0.99), "max_latency_s": lat[-1],
        "mean_queue_s": statistics.mean(r["queue_s"] for r in results),
        "throughput_residues_per_hour": 3600.0 * residues / makespan,
        "throughput_requests_per_s": len(reqs) / makespan, "makespan_s": makespan,
        "peak_running": stats["peak_running"], "peak_gb_in_use": stats["peak_bytes_in_use"] / 1e9,
        "completed": stats["completed"], "failed": stats["failed"], "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    eng.close()


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
    ap.add_argument("--serve", action="store_true", help="run the serving stream instead")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--serve-gap", type=float, default=2.0)
    ap.add_argument("--serve-time-scale", type=float, default=1.0)
    ap.add_argument("--serve-budget-gb", type=float, default=120.0)
    ap.add_argument("--serve-slots", type=int, default=8)
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
