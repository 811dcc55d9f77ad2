"""Generates the full-size golden fixtures of tests/golden/ from the reference itself.

Run in a container where the reference tree is mounted (takes 20-40 minutes
on 8 cores):
    make -C oracle ref && python tests/golden/make_full_golden.py [c2] [c3] [c4]

Every relation list here comes from oracle/_ref/libmps_ref.so, i.e. from the
reference's own Math.hpp/Sieve.hpp (segmented_sieve + run_bsgs, threaded over
chunks like run_worker_pool, Worker.hpp:305-367), never from the project's
code.  This mirrors the reference's own self-test, which compares the sorted
relations of a GPU run with those of a CPU run (kaggle/kaggle_run.py:64-95),
at the benchmark configurations' own sizes.  Outputs:

  c2_full.txt.gz   relations.p of b=10, c=111, 10^12 <= p < 10^12 + 10^10,
                   0 <= n < 10^7, n == 4 (mod 6), sorted by p
  c3_full.txt.gz   relations.p of b=2, c=-25, 9.5e13 <= p < 9.5e13 + 2e10,
                   3.6e6 <= n < 5e6, n == 1 (mod 2), sorted by p
  c4_1e8.json      the 64 mixed-batch items (seed 20261203), each over the
                   first 10^8 of its P range, with their sorted relations
  full.json        item, prime count, relation count and md5 of each of the above
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "mass-prime-siever_b200"))
from oracle.oracle import Reference, make_item, relation_lines  # noqa: E402
import workloads  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
C4_PREFIX = 10**8


def _index() -> dict:
    path = os.path.join(OUT, "full.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def _save_index(idx: dict) -> None:
    with open(os.path.join(OUT, "full.json"), "w") as f:
        json.dump(idx, f, indent=1, sort_keys=True)
        f.write("\n")


def single(ref: Reference, name: str, spec: tuple) -> dict:
    b, c, P0, P1, N0, N1, mod, res = spec
    t0 = time.time()
    rels, nprimes = ref.relations(P0, P1, make_item(*spec))
    text = relation_lines(rels)
    with gzip.GzipFile(os.path.join(OUT, f"{name}_full.txt.gz"), "wb", mtime=0) as f:
        f.write(text.encode())
    rec = {"item": list(spec), "primes": nprimes, "relations": len(rels),
           "md5": hashlib.md5(text.encode()).hexdigest(), "seconds": round(time.time() - t0, 1),
           "threads": os.cpu_count()}
    print(f"{name}: {nprimes} primes, {len(rels)} relations, md5 {rec['md5']} ({rec['seconds']} s)", flush=True)
    return rec


def c4(ref: Reference) -> dict:
    t0 = time.time()
    cases = []
    for k, spec in enumerate(workloads.c4_items(max_width=C4_PREFIX)):
        rels, nprimes = ref.relations(spec[2], spec[3], make_item(*spec))
        cases.append({"name": f"c4_{k:02d}", "item": list(spec), "primes": nprimes,
                      "relations": [list(r) for r in rels]})
        print(f"c4_{k:02d}: {nprimes} primes, {len(rels)} relations ({time.time() - t0:.0f} s)", flush=True)
    with open(os.path.join(OUT, "c4_1e8.json"), "w") as f:
        json.dump({"seed": workloads.C4_SEED, "prefix": C4_PREFIX, "cases": cases}, f, indent=0)
        f.write("\n")
    text = "".join(relation_lines(c["relations"]) for c in cases)
    return {"items": len(cases), "prefix": C4_PREFIX, "seed": workloads.C4_SEED,
            "primes": sum(c["primes"] for c in cases), "relations": sum(len(c["relations"]) for c in cases),
            "md5": hashlib.md5(text.encode()).hexdigest(), "seconds": round(time.time() - t0, 1),
            "threads": os.cpu_count()}


def main(argv: list[str]) -> None:
    if not Reference.available():
        sys.exit("oracle/_ref/libmps_ref.so is missing: run `make -C oracle ref` where the reference is mounted")
    want = argv or ["c2", "c3", "c4"]
    ref = Reference()
    for name in want:
        if name in ("c2", "c3"):
            rec = single(ref, name, workloads.SINGLE[name])
        elif name == "c4":
            rec = c4(ref)
        else:
            sys.exit(f"unknown fixture {name}")
        idx = _index()
        idx[name] = rec
        _save_index(idx)


if __name__ == "__main__":
    main(sys.argv[1:])
