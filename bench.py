"""Benchmark: sieved primes/s of the B200 siever.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|c3|c1|c4|c5] [--width W] [--plain] [--no-sub]

Headline (c1-c3; default c2): one step is one pass of the hot path (segment
sieve -> prep -> exact BSGS -> order) over one item's whole P range, through
the C-ABI (mps_item_relations).  The default item is the plain GPU path at
full size: b=10, c=111, 10^12 <= p < 10^12 + 10^10, 0 <= n < 10^7,
n == 4 (mod 6).  `value` is primes in the range / device time (CUDA events on
the library's streams); `e2e` is the same through the C-ABI with host buffers,
host wall clock.  The relations of the last timed step are compared with the
reference-built fixture (tests/golden/full.json) and the result is `parity`.

With N = 1 and the default workload the line also carries two sub-records:
  batched_vs_plain  the 64-item mixed batch (seed 20261203): the batched
                    engine (mps_batch_relations) against the plain per-item GPU
                    path (each item alone, the reference's plain-method filter,
                    stage-by-stage launches) and against each item alone
                    through the default engine (mps_item_relations);
  served            the served stream (mps_serve_*): Poisson arrivals at
                    0.5x-2x the measured batched capacity, p50/p99 item latency.
--workload c4 / c5 print those records alone.

Under torchrun (N > 1) every rank sieves its own P slice of the same width
(weak scaling, no data-path collective); the per-step time is the max over
ranks.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import math
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
# P width of the CPU baseline's bounded sample per step (the reference's CPU path, all host threads)
CPU_SAMPLE_WIDTH = {"c2": 100_000_000, "c3": 100_000_000, "c1": 99_000_000}
ROOFLINE_WIDTH = 2 * 10**9          # P width of the single-stream per-kernel pass
SERVE_RATES = (0.5, 1.0, 1.5, 2.0)


def relation_text(rels) -> str:
    """relations.p lines "p, M, q" (Worker.hpp:294-297)."""
    return "".join(f"{p}, {M}, {q}\n" for p, M, q in rels)


def golden_index() -> dict:
    try:
        with open(os.path.join(ROOT, "tests", "golden", "full.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def peaks_file():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


# ------------------------------------------------------------------ clocks --

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
        return self

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
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ distributed --

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


def reduce_over_ranks(dist, local: int, value: float, op: str) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist, local: int):
    if dist is not None:
        import torch
        dist.barrier(device_ids=[local])
        torch.cuda.synchronize(local)


# ----------------------------------------------------------- CPU baseline --

def cpu_reference_rate(spec, width: int, threads: int) -> dict:
    """The reference's own segmented_sieve + run_bsgs (oracle/_ref, threaded over
    chunks like run_worker_pool, Worker.hpp:305-367) on [P0, P0 + width).  The
    chunk is a quarter of width / threads (a multiple of 2^20), so that every
    thread stays busy to the end of the sample."""
    from oracle.oracle import Oracle, Reference, make_item as oracle_item
    b, c, P0, _, N0, N1, mod, res, _ = spec
    it = oracle_item(b, c, P0, P0 + width, N0, N1, mod, res)
    chunk = max(1 << 20, (width // (4 * threads)) >> 20 << 20)
    busy = min(threads, -(-width // chunk))
    if Reference.available():
        t0 = time.perf_counter()
        rels, nprimes = Reference().relations(P0, P0 + width, it, threads=threads, chunk=chunk)
        dt = time.perf_counter() - t0
        kind = "reference"
    else:
        orc = Oracle()
        t0 = time.perf_counter()
        rels = orc.relations(P0, P0 + width, it, threads=threads, chunk=chunk)
        dt = time.perf_counter() - t0
        nprimes = len(orc.primes(P0, P0 + width, 1 << 22))
        kind = "port"
    return {"value": nprimes / dt, "primes": nprimes, "seconds": dt, "kind": kind, "relations": len(rels),
            "chunk": chunk, "busy_threads": busy}


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args, spec, label):
    """--impl reference: the reference's own CPU path on all host threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    width = CPU_SAMPLE_WIDTH.get(args.workload, CPU_SAMPLE_WIDTH["c2"])
    if args.width is not None:
        width = min(int(args.width), width)
    for _ in range(args.warmup):
        cpu_reference_rate(spec, max(width // 10, 1 << 22), threads)
    primes_total, secs, kind, busy, chunk = 0, 0.0, "reference", threads, 0
    for _ in range(args.steps):
        r = cpu_reference_rate(spec, width, threads)
        primes_total += r["primes"]
        secs += r["seconds"]
        kind, busy, chunk = r["kind"], r["busy_threads"], r["chunk"]
    value = primes_total / secs
    sample = (f"[P0, P0+{width:.3g}) of the workload per step, {threads} threads over {chunk}-wide chunks "
              f"({busy} busy), {cpu_model()}")
    line = {
        "impl": "reference", "metric": "sieved primes/s", "value": value, "unit": "primes/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": label, "P_width_per_step": width},
        "cpu_baseline": {"value": value, "unit": "primes/s", "cores": threads, "busy_threads": busy, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "primes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------- rooflines --

def sieve_marks_per_odd(hi: int) -> float:
    """Algorithmic bit-marks per odd integer of a segment below hi: the sum of
    1/q over the odd sieving primes q <= 65521 with q*q < hi."""
    lim = min(65536, math.isqrt(hi) + 1)
    comp = bytearray(lim + 1)
    s = 0.0
    for i in range(3, lim + 1, 2):
        if comp[i]:
            continue
        if i * i < hi:
            s += 1.0 / i
        for j in range(i * i, lim + 1, 2 * i):
            comp[j] = 1
    return s


def kernel_rooflines(siever, pieces, peaks, fp64_path: bool) -> dict:
    """Each kernel alone: the chunk path (mps_chunk_relations) runs sieve, prep,
    BSGS and order one after another on one stream, so their CUDA events time
    each kernel without the overlap of the two-slot engine.

    k_bsgs: achieved = BSGS steps (one modular multiply and one table probe or
    insert each, counted on the device) per second; peak = the live-measured
    independent-chain mulmod rate of the same arithmetic without table work.
    k_sieve: achieved = algorithmic bit-marks (sum of 1/q per odd) per second;
    peak = the live-measured conflict-free shared-memory atomicOr rate."""
    tot = {"steps": 0, "baby": 0, "odds": 0, "marks": 0.0, "entries": 0, "survivors": 0,
           "bsgs_ms": 0.0, "sieve_ms": 0.0, "prep_ms": 0.0, "order_ms": 0.0, "launches": 0}
    for lo, hi, item in pieces:
        siever.chunk_relations(lo, hi, item)
        st = siever.stats()
        tot["steps"] += st["bsgs_steps"]
        tot["baby"] += st.get("bsgs_baby_steps", 0)
        tot["odds"] += st["odds"]
        tot["marks"] += st["odds"] * sieve_marks_per_odd(hi)
        tot["entries"] += st["entries"]
        tot["survivors"] += st["survivors"]
        for k in ("bsgs_ms", "sieve_ms", "prep_ms", "order_ms"):
            tot[k] += st[k]
        tot["launches"] += st["bsgs_launches"]
    n = max(tot["launches"], 1)
    mul_peak = peaks["fp64_mulmod_per_s"] if fp64_path else peaks["int_mulmod_per_s"]
    rate = tot["steps"] / (tot["bsgs_ms"] / 1e3) if tot["bsgs_ms"] > 0 else 0.0
    traffic, traffic_src = profile_traffic("k_bsgs")
    hbm = peaks_file().get("hbm_gbs")
    bsgs = {"bound": "alu (fp64-pipe modular multiply + shared-memory table)" if fp64_path
            else "alu (int-pipe Montgomery multiply + shared-memory table)",
            "kernel": "k_bsgs", "achieved": rate / 1e9, "peak": mul_peak / 1e9, "unit": "G mulmod/s",
            "frac": rate / mul_peak if mul_peak else None, "peak_kind": "of measured (live probe)",
            "avg_launch_ms": tot["bsgs_ms"] / n, "steps_per_launch": tot["steps"] / n,
            "baby_steps_per_launch": tot["baby"] / n, "entries_per_launch": tot["entries"] / n,
            "traffic": traffic * tot["steps"] / n if traffic is not None else None,
            "traffic_unit": "DRAM bytes per launch", "traffic_source": traffic_src,
            "hbm_side": {"algorithmic_bytes_per_launch": 72.0 * tot["entries"] / n,
                         "frac_of_measured_hbm": (72.0 * tot["entries"] / (tot["bsgs_ms"] / 1e3)) / (hbm * 1e9)
                         if tot["bsgs_ms"] > 0 and hbm else None},
            "peaks_measured": {k: v / 1e9 for k, v in peaks.items()}}
    smem_peak = peaks.get("smem_atomic_per_s")
    srate = tot["marks"] / (tot["sieve_ms"] / 1e3) if tot["sieve_ms"] > 0 else 0.0
    others = {
        "k_sieve": {"achieved": srate / 1e9, "unit": "G bit-marks/s", "peak": smem_peak / 1e9 if smem_peak else None,
                    "frac": srate / smem_peak if smem_peak else None, "avg_launch_ms": tot["sieve_ms"] / n,
                    "marks_per_launch": tot["marks"] / n, "odds_per_launch": tot["odds"] / n},
        "k_prep": {"avg_launch_ms": tot["prep_ms"] / n, "survivors_per_launch": tot["survivors"] / n,
                   "survivors_per_s": tot["survivors"] / (tot["prep_ms"] / 1e3) if tot["prep_ms"] > 0 else None},
        "k_order": {"avg_launch_ms": tot["order_ms"] / n},
    }
    total_ms = tot["bsgs_ms"] + tot["sieve_ms"] + tot["prep_ms"] + tot["order_ms"]
    shares = {k: tot[k] / total_ms for k in ("sieve_ms", "prep_ms", "bsgs_ms", "order_ms")} if total_ms else {}
    return bsgs, others, shares


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


# ------------------------------------------------------------- sub-records --

def tuning_summary(reports: list[dict], seconds: float) -> dict:
    """The autotuner's choices: how many item classes chose each configuration."""
    counts: dict[str, int] = {}
    for r in reports:
        key = (f"kind{r['table_kind']}" + (f"/load2^-{r['load_shift']}/lanes{r['lanes']}" if r["table_kind"] == 2
                                           else f"/fill{r.get('table_fill', 256)}/scale{r.get('baby_scale', 256)}")
               + f"/ch{r['chains']}/w{r['warps']}/seg{r['seg_words']}")
        counts[key] = counts.get(key, 0) + 1
    gain = [r["default_ns_per_prime"] / r["best_ns_per_prime"] for r in reports if r["best_ns_per_prime"] > 0]
    return {"classes": len(reports), "seconds": seconds, "choices": counts,
            "bsgs_gain_vs_default": {"min": min(gain), "median": statistics.median(gain), "max": max(gain)}
            if gain else None}


def batched_vs_plain(local: int, steps: int, warmup: int, max_width=None, tune: bool = True) -> dict:
    """The 64-item mixed batch (C4): batched engine vs the plain per-item GPU path
    (each item alone, plain-method filter Q = lcm(mod, 2), stage-by-stage
    launches with a host read of each stage's count, one BSGS warp per prime,
    the default launch configuration) vs each item alone through the engine
    with the batched run's tuning.  Same chunk size (2^26 odd numbers)
    everywhere.  Relations must agree exactly."""
    import mps_b200
    import tempfile
    import workloads
    specs = workloads.c4_items(max_width=max_width)
    items = [mps_b200.make_item(*sp) for sp in specs]
    tune_file = os.path.join(tempfile.mkdtemp(prefix="mps_tune_"), "tune.txt")
    with mps_b200.Siever(local) as s:
        nprimes = sum(s.count_primes(sp[2], sp[3]) for sp in specs)
        # one tuning for every path compared (outside every timed region)
        t0 = time.perf_counter()
        reports = s.autotune(items) if tune else []
        tune_s = time.perf_counter() - t0
        s.tune_save(tune_file)

    def open_siever(**kw):
        sv = mps_b200.Siever(local, **kw)
        sv.tune_load(tune_file)
        return sv

    stage = {}

    def batched(s):
        t0 = time.perf_counter()
        r = s.batch_relations(items)
        wall = time.perf_counter() - t0
        st = s.stats()
        stage.update({k: st[k] for k in ("sieve_ms", "prep_ms", "bsgs_ms", "order_ms")})
        return r, st["device_ms"] / 1e3, wall, st["kernel_launches"]

    def per_item(s):
        out, dev, wall, launches = [], 0.0, 0.0, 0
        for k, it in enumerate(items):
            t0 = time.perf_counter()
            r = s.item_relations(it)
            wall += time.perf_counter() - t0
            st = s.stats()
            dev += st["device_ms"] / 1e3
            launches += st["kernel_launches"]
            out += [(k, p, M, q) for p, M, q in r]
        return out, dev, wall, launches

    clocks = ClockSampler(local).start()
    with open_siever() as s:
        for _ in range(warmup):
            batched(s)
        dev_b, wall_b, l_b = 0.0, 0.0, 0
        for _ in range(steps):
            rel_b, d, w, l = batched(s)
            dev_b, wall_b, l_b = dev_b + d, wall_b + w, l_b + l
    short = mps_b200.make_item(*specs[0][:3], specs[0][2] + 10**8, *specs[0][4:])
    # the plain path runs the default launch configuration: the autotuner is part of the batched form
    with mps_b200.Siever(local, plain=1, class_modulus=1) as s:
        for _ in range(warmup):
            s.item_relations(short)
        rel_p, dev_p, wall_p, l_p = per_item(s)
    with open_siever() as s:
        for _ in range(warmup):
            s.item_relations(short)
        rel_a, dev_a, wall_a, l_a = per_item(s)
    clk = clocks.stop()
    parity = "ok" if sorted(rel_b) == sorted(rel_p) == sorted(rel_a) else "mismatch"
    golden = "not checked"
    try:
        with open(os.path.join(ROOT, "tests", "golden", "c4_1e8.json")) as f:
            g = json.load(f)
        golden = "ok"
        for k, case in enumerate(g["cases"]):
            lim = case["item"][3]
            mine = [[p, M, q] for i, p, M, q in rel_b if i == k and p < lim]
            if case["item"][:3] != list(specs[k][:3]) or mine != case["relations"]:
                golden = "mismatch"
                break
    except OSError:
        pass
    b_rate = nprimes * steps / dev_b
    rec = {
        "workload": f"mixed batch: 64 items seed {workloads.C4_SEED}" +
                    (f", P width capped at {max_width:.3g}" if max_width else ", full widths"),
        "primes": nprimes, "relations": len(rel_b),
        "batched": {"value": b_rate, "unit": "primes/s", "ms_per_step": dev_b * 1e3 / steps,
                    "e2e": nprimes * steps / wall_b, "gpu_launches": l_b // steps,
                    "stage_ms_overlapping": stage,
                    "path": "mps_batch_relations: multi-item waves, graph replay, two overlapped slots"},
        "plain_per_item": {"value": nprimes / dev_p, "unit": "primes/s", "ms": dev_p * 1e3, "e2e": nprimes / wall_p,
                           "gpu_launches": l_p,
                           "path": "each item alone, plain-method filter (class_modulus=1: Q = lcm(mod, 2)), "
                                   "stage-by-stage launches, one BSGS warp per prime, 2^26-odd chunks, "
                                   "default launch configuration (not autotuned)"},
        "alone_per_item": {"value": nprimes / dev_a, "unit": "primes/s", "ms": dev_a * 1e3, "e2e": nprimes / wall_a,
                           "gpu_launches": l_a,
                           "path": "each item alone through mps_item_relations, with the batched run's tuning"},
        "ratio_vs_plain": b_rate / (nprimes / dev_p),
        "ratio_vs_alone": b_rate / (nprimes / dev_a),
        "parity": parity, "golden_first_1e8": golden, "clocks": clk,
        "tuning": tuning_summary(reports, tune_s),
    }
    return rec


def served(local: int, duration: float, max_width: int) -> dict:
    """C5: Poisson arrivals of mixed items at multiples of the batched capacity."""
    import mps_b200
    import workloads
    probe = workloads.c4_items(n=32, seed=workloads.C4_SEED + 99, max_width=max_width)
    with mps_b200.Siever(local) as s:
        s.batch_relations([mps_b200.make_item(*x) for x in probe])
        t0 = time.perf_counter()
        s.batch_relations([mps_b200.make_item(*x) for x in probe])
        cap_items = len(probe) / (time.perf_counter() - t0)
        nprimes_probe = sum(s.count_primes(x[2], x[3]) for x in probe)
    results = []
    clocks = ClockSampler(local).start()
    for mult in SERVE_RATES:
        rate = mult * cap_items
        arrivals = workloads.c5_arrivals(rate, duration, max_width=max_width)
        lat, qms = [], []
        with mps_b200.Server(local, max_active=256) as sv:
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
        with mps_b200.Siever(local) as s:
            nprimes = sum(s.count_primes(x[1][2], x[1][3]) for x in arrivals)
        lat.sort()
        pct = (lambda q: lat[min(len(lat) - 1, int(q * len(lat)))]) if lat else (lambda q: None)
        results.append({"load": mult, "arrival_rate_items_s": rate, "items": len(arrivals),
                        "p50_ms": pct(0.50), "p99_ms": pct(0.99),
                        "mean_queue_ms": statistics.mean(qms) if qms else None,
                        "primes_per_s": nprimes / span, "makespan_s": span})
    clk = clocks.stop()
    return {"workload": f"served stream: mixed-batch items, Poisson arrivals, {duration:.0f} s per rate "
                        f"(600 s in the spec, shortened), P width capped at {max_width:.3g}",
            "capacity_items_per_s": cap_items, "capacity_primes_per_s": nprimes_probe * cap_items / len(probe),
            "rates": results, "best_primes_per_s": max(r["primes_per_s"] for r in results), "clocks": clk}


def reference_gpu(local: int, width: int) -> dict:
    """The reference's own GPU worker path on the same GPU: its kernels (psieve,
    prep_sv/prep_svq, bsgs_wg/bsgs_wq, collect, compiled ahead of time from its
    Gpu.hpp by baseline/ref_gpu) driven chunk by chunk as its
    CudaSiever::sieve_filter does, with the flagged numbers checked exactly on
    all host threads (is_prime64 + run_bsgs) while the GPU sieves the next
    chunk.  On [P0, P0 + width) of the default item; relations compared with
    the reference-built fixture."""
    import ctypes
    import gzip
    path = os.path.join(ROOT, "baseline", "_ref", "ref_gpu", "librefgpu.so")
    if not os.path.exists(path):
        return {"unavailable": "baseline/_ref/ref_gpu/librefgpu.so is not built (needs the reference tree)"}
    import mps_b200

    class Item(ctypes.Structure):
        _fields_ = mps_b200.Item._fields_

    class Rel(ctypes.Structure):
        _fields_ = [("p", ctypes.c_uint64), ("M", ctypes.c_uint64), ("q", ctypes.c_uint64)]

    class Stats(ctypes.Structure):
        _fields_ = [("seconds", ctypes.c_double), ("gpu_ms", ctypes.c_double), ("flagged", ctypes.c_uint64),
                    ("declined", ctypes.c_uint64)]

    L = ctypes.CDLL(path)
    L.refgpu_relations.argtypes = [ctypes.c_int, ctypes.POINTER(Item), ctypes.c_uint64, ctypes.c_int,
                                   ctypes.POINTER(Rel), ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t),
                                   ctypes.POINTER(Stats)]
    b, c, P0, _, N0, N1, mod, res, _ = WORKLOADS["c2"]
    it = mps_b200.make_item(b, c, P0, P0 + width, N0, N1, mod, res)
    item = Item(*[getattr(it, f) for f, _ in Item._fields_])
    threads = os.cpu_count() or 1
    chunk = 1 << 28
    cap = 1 << 16
    out = (Rel * cap)()
    n = ctypes.c_size_t()
    st = Stats()
    for _ in range(2):                                     # the second run is kept (the first sets up)
        rc = L.refgpu_relations(local, ctypes.byref(item), chunk, threads, out, cap, ctypes.byref(n), ctypes.byref(st))
        if rc != 0:
            return {"unavailable": f"refgpu_relations returned {rc}"}
    rels = [(out[i].p, out[i].M, out[i].q) for i in range(n.value)]
    with gzip.open(os.path.join(ROOT, "tests", "golden", "c2_full.txt.gz"), "rt") as f:
        want = [tuple(int(x) for x in line.split(",")) for line in f if int(line.split(",")[0]) < P0 + width]
    with mps_b200.Siever(local) as s:
        nprimes = s.count_primes(P0, P0 + width)
    return {"value": nprimes / st.seconds, "unit": "primes/s", "sample": f"[1e12, 1e12+{width:.3g}) of the default item",
            "seconds": st.seconds, "gpu_ms": st.gpu_ms, "cpu_threads": threads, "chunk": chunk,
            "flagged": st.flagged, "declined_chunks": st.declined, "relations": len(rels),
            "parity": "ok" if rels == want else "mismatch",
            "path": "reference kernels (Gpu.hpp) via a restated CudaSiever::sieve_filter, exact CPU check of flagged"}


# -------------------------------------------------------------------- main --

def headline(args, rank, world, local, dist) -> dict:
    import mps_b200
    spec = WORKLOADS[args.workload]
    b, c, P0, width, N0, N1, mod, res, label = spec
    if args.width is not None:
        width = int(args.width)
    lo = P0 + rank * width
    hi = lo + width
    item = mps_b200.make_item(b, c, lo, hi, N0, N1, mod, res)
    siever = mps_b200.Siever(local, plain=1 if args.plain else 0)

    # units: primes in this rank's slice (counted on the device, outside the timed region)
    nprimes = siever.count_primes(lo, hi)
    total_primes = reduce_over_ranks(dist, local, float(nprimes), "sum")
    # the autotuner's choice for this item (outside the timed region)
    t0 = time.perf_counter()
    reports = siever.autotune([item]) if not args.no_tune else []
    tuning = tuning_summary(reports, time.perf_counter() - t0)

    for _ in range(args.warmup):
        siever.item_relations(item)

    clocks = ClockSampler(local)
    barrier(dist, local)
    clocks.start()
    t0 = time.perf_counter()
    acc = {"device_ms": 0.0, "sieve_ms": 0.0, "prep_ms": 0.0, "bsgs_ms": 0.0, "order_ms": 0.0,
           "kernel_launches": 0}
    rels, entries = [], 0
    for _ in range(args.steps):
        rels = siever.item_relations(item)
        st = siever.stats()
        for k in acc:
            acc[k] += st[k]
        entries = st["entries"]
    wall = time.perf_counter() - t0
    barrier(dist, local)
    clk = clocks.stop()

    dev_s = reduce_over_ranks(dist, local, acc["device_ms"] / 1e3, "max")
    wall_s = reduce_over_ranks(dist, local, wall, "max")
    value = total_primes * args.steps / dev_s
    e2e = total_primes * args.steps / wall_s

    parity = "not checked (no fixture for this range)"
    g = golden_index().get(args.workload)
    if g and g["item"] == [b, c, lo, hi, N0, N1, mod, res]:
        ok = hashlib.md5(relation_text(rels).encode()).hexdigest() == g["md5"] and len(rels) == g["relations"]
        parity = "ok" if ok else "mismatch"

    peaks = siever.measure_peaks()
    fp64_path = hi <= (1 << 49)
    rw = min(width, ROOFLINE_WIDTH)
    roof, kernels, shares = kernel_rooflines(
        siever, [(lo, lo + rw, mps_b200.make_item(b, c, lo, lo + rw, N0, N1, mod, res))], peaks, fp64_path)
    roof["sample"] = f"[P0, P0+{rw:.3g}) of this rank's slice, one chunk per launch, one stream"

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cw = CPU_SAMPLE_WIDTH[args.workload]
        r = cpu_reference_rate(spec, cw, threads)
        cpu = {"value": r["value"], "unit": "primes/s", "cores": threads, "busy_threads": r["busy_threads"],
               "kind": r["kind"],
               "sample": f"[{P0:.4g}, {P0:.4g}+{cw:.3g}) of the same item ({r['primes']} primes, "
                         f"{r['seconds']:.1f} s, {r['chunk']}-wide chunks), {cpu_model()}"}
    siever.close()
    steps = args.steps
    return {
        "metric": "sieved primes/s", "value": value, "unit": "primes/s", "n_gpus": world,
        "steps": steps, "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic",
        "config": {"workload": label, "P_width_per_gpu": width, "path": "plain" if args.plain else "persistent",
                   "l2": "working set (survivors, entries) > 126 MB L2 per chunk; no flush"},
        "e2e": {"value": e2e, "unit": "primes/s", "h2d_bytes_per_step": 112, "d2h_bytes_per_step": 24 * len(rels)},
        "gpu_launches": acc["kernel_launches"], "relations": len(rels), "parity": parity,
        "bsgs_primes": entries, "primes": int(total_primes),
        "stage_ms_per_step": {k: acc[k] / steps for k in ("sieve_ms", "prep_ms", "bsgs_ms", "order_ms")},
        "roofline": roof, "kernels": kernels, "single_stream_shares": shares, "tuning": tuning,
        "cpu_baseline": cpu, "clocks": clk,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS) + ["c4", "c5", "refgpu"])
    ap.add_argument("--duration", type=float, default=10.0, help="served: seconds of arrivals per rate")
    ap.add_argument("--serve-width", type=float, default=1e9, help="served: P width cap per item")
    ap.add_argument("--width", type=float, default=None, help="P width per rank (default: the workload's)")
    ap.add_argument("--plain", action="store_true", help="the plain per-chunk path")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="run the default configuration instead of the tuned one")
    ap.add_argument("--no-sub", action="store_true", help="skip the batched, served and reference-GPU sub-records")
    args = ap.parse_args()

    if args.impl == "reference":
        spec = WORKLOADS["c2" if args.workload in ("c4", "c5", "refgpu") else args.workload]
        return run_reference(args, spec, spec[-1])

    rank, world, local, dist = dist_setup(args.gpus)
    if args.workload == "refgpu":
        if rank == 0:
            print(json.dumps(reference_gpu(local, int(args.width) if args.width else 10**9)), flush=True)
        return 0
    if args.workload in ("c4", "c5"):
        if rank == 0:
            if args.workload == "c4":
                rec = batched_vs_plain(local, args.steps, min(args.warmup, 1),
                                       int(args.width) if args.width else None, tune=not args.no_tune)
            else:
                rec = served(local, args.duration, int(args.serve_width))
            print(json.dumps(rec), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return 0

    line = headline(args, rank, world, local, dist)
    if world == 1 and args.workload == "c2" and args.width is None and not args.no_sub:
        line["batched_vs_plain"] = batched_vs_plain(local, 1, 1, tune=not args.no_tune)
        line["served"] = served(local, args.duration, int(args.serve_width))
        line["reference_gpu"] = reference_gpu(local, 10**9)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
