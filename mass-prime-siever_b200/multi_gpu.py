"""P-range sharding over several GPUs: one process per GPU, no data-path collective.

The reference runs one siever process per GPU on its own slice of [P0, P1)
(kaggle/kaggle_run.py:155-176: step = (P1 - P0) // n, the last slice takes
the rest) and merges the runs' results.json files afterwards by intersecting
their "prp" lists (kaggle/merge_results.py:16-52).  Here the same split runs
under torch.distributed (one rank per GPU, launched by torchrun): every rank
sieves its slice on its own GPU, and the only exchange is one gather of the
relations (24 bytes per relation) to rank 0, which writes relations.p in
increasing p and the item's results.json entry through the drop-in program.

    torchrun --nproc-per-node N --master-addr 127.0.0.1 mass-prime-siever_b200/multi_gpu.py \\
        --item "Factor=2,-25,1000000000000,2000000000000,3600000,5000000,2,1" --out run_dir

merge_results() restates merge_results.py for results files of separate runs.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def parse_factor_line(line: str) -> tuple:
    """`Factor=b,c,P0,P1,N0,N1[,mod,res]` (Config.hpp:124-200) -> 8-tuple."""
    line = line.strip()
    if line.startswith("Factor="):
        line = line[len("Factor="):]
    parts = [p.strip() for p in line.split(",") if p.strip()]
    if len(parts) not in (6, 8):
        raise ValueError("must have 6 or 8 comma-separated values (b,c,P0,P1,N0,N1[,mod,res])")
    vals = [int(p) for p in parts]
    if len(vals) == 6:
        vals += [1, 0]
    b, c, P0, P1, N0, N1, mod, res = vals
    if mod == 0 or not 0 <= res < mod:
        raise ValueError("class must satisfy 0 <= res < mod")
    if P0 >= P1 or N0 >= N1:
        raise ValueError("requires P0 < P1 and N0 < N1")
    return b, c, P0, P1, N0, N1, mod, res


def factor_line(spec: tuple) -> str:
    b, c, P0, P1, N0, N1, mod, res = spec
    return f"Factor={b},{c},{P0},{P1},{N0},{N1},{mod},{res}"


def shard_bounds(P0: int, P1: int, world: int, rank: int) -> tuple[int, int]:
    """Rank `rank`'s slice of [P0, P1) (kaggle_run.py:155-161)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    step = (P1 - P0) // world
    lo = P0 + rank * step
    hi = P1 if rank == world - 1 else lo + step
    return lo, hi


def slice_relations(compute, spec: tuple, world: int, rank: int) -> list[tuple[int, int, int]]:
    """This rank's relations: compute(lo, hi, spec) on its slice, or [] when
    the slice is empty (a P range narrower than the world size), so that
    every rank still reaches the gather."""
    lo, hi = shard_bounds(spec[2], spec[3], world, rank)
    return compute(lo, hi, spec) if lo < hi else []


def merge_relations(parts: list[list[tuple[int, int, int]]]) -> list[tuple[int, int, int]]:
    """Concatenate per-rank relations (disjoint P slices) in increasing p."""
    out = sorted(r for part in parts for r in part)
    for a, b in zip(out, out[1:]):
        if a[0] == b[0]:
            raise ValueError(f"prime {a[0]} reported by two shards")
    return out


def gather_relations(dist, rels: list[tuple[int, int, int]], rank: int, world: int):
    """Every rank's relations to rank 0 (None on the other ranks).  Works on
    gloo (CPU) and nccl; the objects are small lists of (p, M, q)."""
    if dist is None or world == 1:
        return merge_relations([rels])
    parts = [None] * world if rank == 0 else None
    dist.gather_object(rels, parts, dst=0)
    return merge_relations(parts) if rank == 0 else None


def merge_results(entries_per_file: list[list[dict]]) -> dict:
    """merge_results.py:16-52: the n left after all runs are the n listed as
    "prp" in every entry (same b, c, N0, N1 required); also the P ranges
    covered and the gaps between them."""
    survivors, key, ranges = None, None, []
    for fi, entries in enumerate(entries_per_file):
        for e in entries:
            this = (int(e["b"]), int(e["c"]), int(e["N0"]), int(e["N1"]))
            if key is None:
                key = this
            elif this != key:
                raise ValueError(f"file {fi}: b, c, N0, N1 = {this} differ from {key}; not merging")
            prp = {int(n) for n in e["prp"]}
            survivors = prp if survivors is None else survivors & prp
            ranges.append((int(e["P0"]), int(e["P1"]), fi))
    ranges.sort()
    gaps = [(a1, b0) for (_, a1, _), (b0, _, _) in zip(ranges, ranges[1:]) if b0 > a1]
    return {"key": key, "survivors": sorted(survivors or ()), "ranges": ranges, "gaps": gaps}


def write_outputs(out_dir: str, spec: tuple, rels: list[tuple[int, int, int]], siever_bin: str | None = None):
    """relations.p (increasing p) and the results.json entry of the whole
    item, the latter through the drop-in program's own writer."""
    os.makedirs(out_dir, exist_ok=True)
    rp = os.path.join(out_dir, "relations.p")
    with open(rp, "w") as f:
        f.writelines(f"{p}, {M}, {q}\n" for p, M, q in rels)
    siever_bin = siever_bin or os.path.join(HERE, "mps_siever")
    ts = time.strftime("%Y-%m-%d %H:%M:%S UTC+0", time.gmtime())
    subprocess.run([siever_bin, "--results-entry", rp, factor_line(spec), ts, os.path.join(out_dir, "results.json")],
                   check=True, stdout=subprocess.DEVNULL)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--item", required=True, help="a worktodo line, Factor=b,c,P0,P1,N0,N1[,mod,res]")
    ap.add_argument("--out", default=".")
    args = ap.parse_args(argv)
    spec = parse_factor_line(args.item)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import mps_b200

    def on_gpu(lo, hi, sp):
        b, c, _, _, N0, N1, mod, res = sp
        with mps_b200.Siever(local) as s:
            return s.item_relations(mps_b200.make_item(b, c, lo, hi, N0, N1, mod, res))

    t0 = time.perf_counter()
    rels = slice_relations(on_gpu, spec, world, rank)
    dt = time.perf_counter() - t0
    merged = gather_relations(dist, rels, rank, world)
    if rank == 0:
        write_outputs(args.out, spec, merged)
        print(json.dumps({"item": factor_line(spec), "ranks": world, "relations": len(merged),
                          "rank0_seconds": dt}), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
