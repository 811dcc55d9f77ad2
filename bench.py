"""Benchmark: sieved primes/s of the B200 siever.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|c3|c1|c4|c5] [--width W] [--plain]

c1-c3: one step is one pass of the hot path (segment sieve -> prep -> exact
BSGS -> order) over one item's whole P range, through the C-ABI
(mps_item_relations).  Default workload (the plain GPU path, full size):
b=10, c=111, 10^12 <= p < 10^12 + 10^10, 0 <= n < 10^7, n == 4 (mod 6).
c4: one step is the 64-item mixed batch through mps_batch_relations (the
batched engine); the plain per-item path is timed once beside it.
c5: the served stream (mps_serve_*): Poisson arrivals at 0.5x-2x the measured
batched capacity; p50/p99 item latency per rate.

Under torchrun (N > 1) every rank sieves its own P slice of the same width
(weak scaling, no data-path collective); the per-step time is the max over
ranks.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "mass-prime-siever_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

WORKLOADS = {
    # name: (b, c, P0, width, N0, N1, mod, res, label)
    "c2": (10, 111, 10**12, 10**10, 0, 10**7, 6, 4,
           "plain GPU path, full size: b=10 c=111 p in [1e12, 1e12+1e10) n in [0, 1e7) n==4 mod 6"),
    "c3": (2, -25, 95 * 10**12, 2 * 10**10, 3_600_000, 5_000_000, 2, 1,
           "residue classes: b=2 c=-25 p in [9.5e13, 9.5e13+2e10) n in [3.6e6, 5e6) n==1 mod 2"),
    "c1": (2, -25, 10**6, 10**8 - 10**6, 0, 100_000, 2, 1,
           "small CPU-runnable: b=2 c=-25 p in [1e6, 1e8) n in [0, 1e5) n==1 mod 2"),
}
CPU_SAMPLE_WIDTH = {"c2": 30_000_000, "c3": 20_000_000, "c1": 99_000_000}
ROOFLINE_WIDTH = 2 * 10**9          # P width of the k_bsgs roofline pass


def run_batch(args, siever_cls, make_item, workloads, rank, world, local, dist):
    """c4: the mixed batch, batched engine vs the plain per-item path."""
    import mps_b200
    specs = workloads.c4_items(max_width=int(args.width) if args.width else None)
    items = [make_item(*sp) for sp in specs]
    with mps_b200.Siever(local) as counter:
        nprimes = sum(counter.count_primes(sp[2], sp[3]) for sp in specs)
    total_primes = sum_over_ranks(dist, local, float(nprimes))

    def timed(siever, steps, warmup):
        for _ in range(warmup):
            siever.batch_relations(items)
        dev, wall, launches, rels = 0.0, 0.0, 0, 0
        bsgs_ms, bsgs_steps = 0.0, 0
        for _ in range(steps):
            t0 = time.perf_counter()
            r = siever.batch_relations(items)
            wall += time.perf_counter() - t0
            st = siever.stats()
            dev += st["device_ms"] / 1e3
            launches += st["kernel_launches"]
            bsgs_ms += st["bsgs_ms"]
            bsgs_steps += st["bsgs_steps"]
            rels = len(r)
        return dev, wall, launches, rels, bsgs_ms, bsgs_steps

    batched = mps_b200.Siever(local)
    clocks = ClockSampler(local)
    barrier(dist, local)
    clocks.start()
    dev, wall, launches, rels, bsgs_ms, bsgs_steps = timed(batched, args.steps, args.warmup)
    barrier(dist, local)
    clk = clocks.stop()
    peaks = batched.measure_peaks()
    batched.close()
    plain = mps_b200.Siever(local, plain=1, chunk_odds=1 << 23)
    pdev, pwall, plaunches, prels, _, _ = timed(plain, 1, 1)
    plain.close()
    if prels != rels:
        raise RuntimeError("plain and batched relation counts differ")
    dev = max_over_ranks(dist, local, dev)
    wall = max_over_ranks(dist, local, wall)
    pdev = max_over_ranks(dist, local, pdev)
    value = total_primes * args.steps / dev
    with mps_b200.Siever(local) as rs:
        pieces = [(sp[2], min(sp[3], sp[2] + 10**8), make_item(*sp[:3], min(sp[3], sp[2] + 10**8), *sp[4:]))
                  for sp in specs]
        roofline = bsgs_roofline(rs, pieces, peaks, all(sp[3] <= (1 << 49) for sp in specs))
    roofline["sample"] = "the first 1e8 of every item, one chunk per launch, one stream"
    if rank == 0:
        line = {
            "metric": "sieved primes/s", "value": value, "unit": "primes/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": f"mixed batch: 64 items seed {workloads.C4_SEED}" +
                                   (f", P width capped at {args.width:.3g}" if args.width else ", full widths"),
                       "path": "batched (multi-item waves, graph replay, two overlapped slots)",
                       "l2": "working set per wave > 126 MB L2; no flush"},
            "plain_per_item": {"value": total_primes / pdev, "unit": "primes/s", "ms_per_step": pdev * 1e3,
                               "path": "one item after another, 2^23-odd chunks, host sync per stage",
                               "kernel_launches": plaunches},
            "e2e": {"value": total_primes * args.steps / wall, "unit": "primes/s",
                    "h2d_bytes_per_step": 112 * len(items), "d2h_bytes_per_step": 28 * rels},
            "gpu_launches": launches, "relations": rels, "primes": int(total_primes),
            "roofline": roofline,
            "cpu_baseline": None, "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    return 0


def run_serve(args, rank):
    """c5: Poisson arrivals of mixed items at multiples of the batched capacity."""
    import mps_b200
    import workloads
    if rank != 0:
        return 0
    cap_w = int(args.width) if args.width else 10**9
    duration = args.duration
    # capacity: items/s of the batched engine on mixed items of the same distribution
    probe = workloads.c4_items(n=32, seed=workloads.C4_SEED + 99, max_width=cap_w)
    with mps_b200.Siever(0) as s:
        s.batch_relations([mps_b200.make_item(*x) for x in probe])
        t0 = time.perf_counter()
        s.batch_relations([mps_b200.make_item(*x) for x in probe])
        cap_items = len(probe) / (time.perf_counter() - t0)
        nprimes_probe = sum(s.count_primes(x[2], x[3]) for x in probe)
    results = []
    clocks = ClockSampler(0)
    clocks.start()
    for mult in (0.5, 1.0, 1.5, 2.0):
        rate = mult * cap_items
        arrivals = workloads.c5_arrivals(rate, duration, max_width=cap_w)
        lat, qms = [], []
        with mps_b200.Server(0, max_active=256) as sv:
            t_start = time.perf_counter()
            tickets = []
            for t_arr, spec in arrivals:
                now = time.perf_counter() - t_start
                if t_arr > now:
                    time.sleep(t_arr - now)
                tickets.append(sv.submit(mps_b200.make_item(*spec)))
            for t in tickets:
                st = sv.wait(t, timeout=3600)
                lat.append(st["latency_ms"])
                qms.append(st["queue_ms"])
            span = time.perf_counter() - t_start
        with mps_b200.Siever(0) as s:
            nprimes = sum(s.count_primes(x[1][2], x[1][3]) for x in arrivals)
        lat.sort()
        pct = lambda q: lat[min(len(lat) - 1, int(q * len(lat)))] if lat else None
        results.append({"load": mult, "arrival_rate_items_s": rate, "items": len(arrivals),
                        "p50_ms": pct(0.50), "p99_ms": pct(0.99), "mean_queue_ms": statistics.mean(qms) if qms else None,
                        "primes_per_s": nprimes / span, "makespan_s": span})
    clk = clocks.stop()
    best = max(r["primes_per_s"] for r in results)
    line = {
        "metric": "sieved primes/s (served) with p50/p99 item latency", "value": best, "unit": "primes/s",
        "n_gpus": 1, "steps": len(results), "warmup": 1, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": f"served stream: c4-distributed items, Poisson arrivals, {duration:.0f} s per rate "
                               f"(600 s in the spec, shortened), P width capped at {cap_w:.3g}",
                   "capacity_items_per_s": cap_items, "capacity_primes_per_s": nprimes_probe * cap_items / len(probe)},
        "rates": results,
        "e2e": {"value": best, "unit": "primes/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    return 0


def profile_traffic(kernel: str):
    """DRAM bytes per BSGS step of `kernel` from the committed ncu summary
    (profiles/traffic.txt lines: "<kernel> <bytes per step> <source ...>")."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.txt")) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and parts[0] == kernel and not line.startswith("#"):
                    return float(parts[1]), " ".join(parts[2:])
    except OSError:
        pass
    return None, None


def bsgs_roofline(siever, pieces, peaks, fp64_path: bool) -> dict:
    """k_bsgs alone: the same persistent kernel launched one chunk at a time on
    one stream (mps_chunk_relations), so its CUDA events time it without the
    overlap of the two-slot engine.  achieved = BSGS steps (one modular
    multiply and one table operation each, counted on the device) per second
    of k_bsgs launch time; peak = the live-measured mulmod rate of the same
    arithmetic without table work."""
    steps, ms, launches, entries = 0, 0.0, 0, 0
    for lo, hi, item in pieces:
        siever.chunk_relations(lo, hi, item)
        st = siever.stats()
        steps += st["bsgs_steps"]
        ms += st["bsgs_ms"]
        launches += st["bsgs_launches"]
        entries += st["entries"]
    mul_peak = peaks["fp64_mulmod_per_s"] if fp64_path else peaks["int_mulmod_per_s"]
    rate = steps / (ms / 1e3) if ms > 0 else 0.0
    per_step, src = profile_traffic("k_bsgs")
    steps_per_launch = steps / launches if launches else 0
    hbm = peaks_file().get("hbm_gbs")
    return {"bound": "alu (fp64-pipe modular multiply + shared-memory table)" if fp64_path
            else "alu (int-pipe Montgomery multiply + shared-memory table)",
            "kernel": "k_bsgs", "achieved": rate / 1e9, "peak": mul_peak / 1e9, "unit": "G mulmod/s",
            "frac": rate / mul_peak if mul_peak else None,
            "avg_launch_ms": ms / launches if launches else None, "steps_per_launch": steps_per_launch,
            "traffic": per_step * steps_per_launch if per_step is not None else None,
            "traffic_unit": "DRAM bytes per launch", "traffic_source": src,
            "peak_source": "measured live (mps_measure_peaks): independent-chain mulmod probe, same arithmetic",
            "peaks_measured": {k: v / 1e9 for k, v in peaks.items()},
            "hbm_side": {"algorithmic_bytes_per_launch": 72.0 * entries / launches if launches else None,
                         "note": "72 B entry read per prime; relations are a few bytes per launch",
                         "frac_of_measured_hbm": (72.0 * entries / (ms / 1e3)) / (hbm * 1e9) if ms > 0 and hbm
                         else None}}


def peaks_file():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


class ClockSampler:
    """nvidia-smi samples (SM clock, throttle reasons) during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.reader.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        return rank, world, local, dist
    return 0, 1, 0, None


def max_over_ranks(dist, local: int, value: float) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, local: int, value: float) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist, local: int):
    if dist is not None:
        import torch
        dist.barrier(device_ids=[local])
        torch.cuda.synchronize(local)


def cpu_reference_rate(spec, width: int, threads: int):
    """The reference's own segmented_sieve + run_bsgs (oracle/_ref, threaded like
    run_worker_pool) on [P0, P0 + width): (primes/s, primes, seconds, kind)."""
    from oracle.oracle import Oracle, Reference, make_item as oracle_item
    b, c, P0, _, N0, N1, mod, res, _ = spec
    it = oracle_item(b, c, P0, P0 + width, N0, N1, mod, res)
    if Reference.available():
        ref = Reference()
        t0 = time.perf_counter()
        rels, nprimes = ref.relations(P0, P0 + width, it, threads=threads)
        dt = time.perf_counter() - t0
        return nprimes / dt, nprimes, dt, "reference", len(rels)
    orc = Oracle()
    t0 = time.perf_counter()
    rels = orc.relations(P0, P0 + width, it, threads=threads)
    dt = time.perf_counter() - t0
    nprimes = len(orc.primes(P0, P0 + width, 1 << 22))
    return nprimes / dt, nprimes, dt, "port", len(rels)


def run_reference(args, spec, label):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    width = CPU_SAMPLE_WIDTH[args.workload] if args.width is None else min(int(args.width), CPU_SAMPLE_WIDTH[args.workload])
    for _ in range(args.warmup):
        cpu_reference_rate(spec, max(width // 10, 1_000_000), threads)
    rates, primes_total, secs = [], 0, 0.0
    kind = "reference"
    for _ in range(args.steps):
        rate, nprimes, dt, kind, _ = cpu_reference_rate(spec, width, threads)
        rates.append(rate)
        primes_total += nprimes
        secs += dt
    value = primes_total / secs
    sample = f"[P0, P0+{width:.3g}) of the workload per step, {threads} threads"
    line = {
        "impl": "reference", "metric": "sieved primes/s", "value": value, "unit": "primes/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": label, "P_width_per_step": width},
        "cpu_baseline": {"value": value, "unit": "primes/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "primes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS) + ["c4", "c5"])
    ap.add_argument("--duration", type=float, default=15.0, help="c5: seconds of arrivals per rate")
    ap.add_argument("--width", type=float, default=None, help="P width per rank (default: the workload's)")
    ap.add_argument("--plain", action="store_true", help="the plain per-chunk path")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.workload in ("c4", "c5"):
        if args.impl == "reference":
            spec = WORKLOADS["c2"]
            return run_reference(args, spec, spec[-1])
        rank, world, local, dist = dist_setup(args.gpus)
        import mps_b200
        import workloads
        if args.workload == "c5":
            return run_serve(args, rank)
        rc = run_batch(args, mps_b200.Siever, mps_b200.make_item, workloads, rank, world, local, dist)
        if dist is not None:
            dist.destroy_process_group()
        return rc
    spec = WORKLOADS[args.workload]
    b, c, P0, width, N0, N1, mod, res, label = spec
    if args.width is not None:
        width = int(args.width)

    if args.impl == "reference":
        return run_reference(args, spec, label)

    rank, world, local, dist = dist_setup(args.gpus)
    import mps_b200
    lo = P0 + rank * width
    hi = lo + width
    item = mps_b200.make_item(b, c, lo, hi, N0, N1, mod, res)
    siever = mps_b200.Siever(local, plain=1 if args.plain else 0)

    # units: primes in this rank's slice (counted on the device, outside the timed region)
    nprimes = siever.count_primes(lo, hi)
    total_primes = sum_over_ranks(dist, local, float(nprimes))

    for _ in range(args.warmup):
        siever.item_relations(item)

    clocks = ClockSampler(local)
    barrier(dist, local)
    clocks.start()
    t0 = time.perf_counter()
    dev_ms, bsgs_ms, steps_done, launches, rel_count, entries = 0.0, 0.0, 0, 0, 0, 0
    for _ in range(args.steps):
        rels = siever.item_relations(item)
        st = siever.stats()
        dev_ms += st["device_ms"]
        bsgs_ms += st["bsgs_ms"]
        steps_done += st["bsgs_steps"]
        launches += st["kernel_launches"]
        rel_count = len(rels)
        entries = st["entries"]
    wall = time.perf_counter() - t0
    barrier(dist, local)
    clk = clocks.stop()

    dev_s = max_over_ranks(dist, local, dev_ms / 1e3)
    wall_s = max_over_ranks(dist, local, wall)
    value = total_primes * args.steps / dev_s
    e2e = total_primes * args.steps / wall_s

    peaks = siever.measure_peaks()
    fp64_path = hi <= (1 << 49)
    rw = min(width, ROOFLINE_WIDTH)
    roofline = bsgs_roofline(siever, [(lo, lo + rw, mps_b200.make_item(b, c, lo, lo + rw, N0, N1, mod, res))],
                             peaks, fp64_path)
    roofline["sample"] = f"[P0, P0+{rw:.3g}) of this rank's slice, one chunk per launch, one stream"

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cw = CPU_SAMPLE_WIDTH[args.workload]
        rate, np_, dt, kind, _ = cpu_reference_rate(spec, cw, threads)
        cpu = {"value": rate, "unit": "primes/s", "cores": threads, "kind": kind,
               "sample": f"[{P0:.4g}, {P0:.4g}+{cw:.3g}) of the same item ({np_} primes, {dt:.1f} s)"}

    if rank == 0:
        line = {
            "metric": "sieved primes/s", "value": value, "unit": "primes/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic",
            "config": {"workload": label, "P_width_per_gpu": width, "path": "plain" if args.plain else "persistent",
                       "l2": "working set (survivors, entries) > 126 MB L2 per chunk; no flush"},
            "e2e": {"value": e2e, "unit": "primes/s", "h2d_bytes_per_step": 112,
                    "d2h_bytes_per_step": 24 * rel_count},
            "gpu_launches": launches,
            "relations": rel_count, "bsgs_primes": entries, "primes": int(total_primes),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    siever.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
