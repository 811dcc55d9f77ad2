"""Generates the golden fixtures of tests/golden/ from the reference itself.

Run in a container where the reference tree is mounted:
    make -C oracle ref && python tests/golden/make_golden.py

Every relation list here comes from oracle/_ref/libmps_ref.so, i.e. from the
reference's own Math.hpp/Sieve.hpp (segmented_sieve + run_bsgs, threaded
like run_worker_pool), never from the project's code.  Outputs:

  relations.json       items with their sorted relations.p lines
  c1_relations.txt.gz  the full relations of the small CPU-runnable config
                       (b=2, c=-25, 10^6 <= p < 10^8, 0 <= n < 10^5, 2/1)
  is_prime.json        is_prime64 verdicts, incl. strong pseudoprimes
  single_primes.json   run_bsgs of single primes with degenerate orders
"""
from __future__ import annotations

import gzip
import hashlib
import json
import math
import os
import random
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.oracle import Reference, make_item, relation_lines  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
SEED = 20261203

# (name, b, c, P0, P1, N0, N1, mod, res)
ITEMS = [
    # kaggle/kaggle_run.py:66 self-test item (GPU == CPU sorted relations)
    ("selftest", 2, -25, 10_000_000_000, 10_020_000_000, 3_600_000, 5_000_000, 2, 1),
    # 10^n + 111 class 4 mod 6 (the second README example), dense slice at low p
    ("c2_low", 10, 111, 1_000_000_000, 1_030_000_000, 0, 10_000_000, 6, 4),
    # the plain full-size item, first 3e7 of its P range
    ("c2_slice", 10, 111, 10**12, 10**12 + 30_000_000, 0, 10_000_000, 6, 4),
    # the residue-class item at lower p (dense) and a slice at its own p
    ("c3_low", 2, -25, 10**10, 10**10 + 50_000_000, 3_600_000, 5_000_000, 2, 1),
    ("c3_slice", 2, -25, 95 * 10**12, 95 * 10**12 + 20_000_000, 3_600_000, 5_000_000, 2, 1),
    # no class, odd b and the 12/7 class (the survey's probe items), narrowed
    ("b7_nomod", 7, -3, 5_000_000_000, 5_005_000_000, 0, 1_000_000, 1, 0),
    ("b12_mod12", 12, 5, 5_000_000_000, 5_020_000_000, 0, 1_000_000, 12, 7),
    # small primes: p < 1000 goes through run_bsgs_reference (Math.hpp:488-542)
    ("small_p_2", 2, -25, 2, 300_000, 0, 1_000, 1, 0),
    ("small_p_10", 10, 111, 2, 200_000, 0, 2_000, 6, 4),
    ("small_p_negb", -3, 7, 2, 50_000, 0, 500, 2, 0),
    # p | b (b prime in range) with p | c (relation p, N0, 1) and without
    ("p_div_b_and_c", 1_000_003, -2_000_006, 999_000, 1_001_000, 5, 50, 1, 0),
    ("p_div_b_only", 1_000_003, 7, 999_000, 1_001_000, 5, 50, 1, 0),
    ("p_div_c_only", 3, -1_000_003, 999_000, 1_001_000, 0, 5_000, 1, 0),
    # c beyond 64 bits (b and c are 128-bit integers in the reference)
    ("c_128bit", 2, (1 << 70) + 1, 10**9, 10**9 + 2_000_000, 0, 100_000, 1, 0),
    ("b_128bit", (1 << 80) + 3, -1, 10**9, 10**9 + 1_000_000, 1, 50_000, 2, 0),
    # N ranges: N0 > 0 with a narrow window, n_start >= N1 (no work), mod > span
    ("narrow_n", 10, -7, 10**9, 10**9 + 3_000_000, 999_990, 1_000_010, 12, 11),
    ("empty_class", 5, 2, 10**9, 10**9 + 100_000, 10, 12, 12, 0),
    ("mod_gt_span", 6, 1, 10**9, 10**9 + 2_000_000, 100, 130, 48, 10),
    # widest N range (10^7) with no class: the largest baby-step tables
    ("wide_n", 3, 2, 10**11, 10**11 + 2_000_000, 0, 10_000_000, 1, 0),
    # odd class modulus and the largest even one used by the class split (48)
    ("mod3", 5, -4, 10**9, 10**9 + 5_000_000, 0, 1_000_000, 3, 2),
    ("mod48", 6, 5, 10**9, 10**9 + 5_000_000, 0, 5_000_000, 48, 5),
]


def c4_items(n: int, seed: int, pwidth: int):
    """Items drawn like the 64-item mixed batch (b, c, P0, N0, N width, mod, res),
    with a fixed narrow P width so the reference finishes in seconds."""
    rng = random.Random(seed)
    out = []
    while len(out) < n:
        b = rng.choice([2, 3, 5, 6, 7, 10, 12])
        c = rng.choice([x for x in range(-999, 1000) if x != 0])
        if math.gcd(b, abs(c)) != 1:
            continue
        P0 = int(10 ** rng.uniform(9, 14))
        N0 = rng.randint(0, 10**6)
        NW = int(10 ** rng.uniform(4, 7))
        mod = rng.choice([1, 2, 6, 12])
        res = rng.randrange(mod)
        out.append((f"c4_{len(out):02d}", b, c, P0, P0 + pwidth, N0, N0 + NW, mod, res))
    return out


IS_PRIME_CASES = [
    0, 1, 2, 3, 4, 5, 9, 25, 37, 41, 561, 1105, 1729, 2047, 3277, 4033, 4681, 8321,
    1_373_653, 25_326_001, 3_215_031_751, 2_152_302_898_747, 3_474_749_660_383,
    341_550_071_728_321, 3_825_123_056_546_413_051, 318_665_857_834_031_151_167_461 % (1 << 64),
    4_294_967_291, 4_294_967_297, 65_521 * 65_521, 65_537 * 65_537, 4_611_686_018_427_387_847,
    (1 << 61) - 1, (1 << 62) - 57, (1 << 62) - 1, (1 << 64) - 59, (1 << 64) - 1,
    1_111_111_111_111_111_111, 999_999_999_989, 1_000_000_000_039,
]


def strong_pseudoprimes_base2(limit: int):
    """Odd composites n < limit that are strong probable primes to base 2."""
    out = []
    for n in range(5, limit, 2):
        d, s = n - 1, 0
        while d % 2 == 0:
            d //= 2
            s += 1
        x = pow(2, d, n)
        if x in (1, n - 1) or any(pow(x, 1 << r, n) == n - 1 for r in range(1, s)):
            if any(n % q == 0 for q in range(3, int(n**0.5) + 1, 2)):
                out.append(n)
    return out


def carmichael_like(count: int, seed: int):
    """Products (k+1)(2k+1) and (6k+1)(12k+1)(18k+1) near 2^62 (hard MR inputs)."""
    rng = random.Random(seed)
    out = []
    while len(out) < count:
        k = rng.randrange(1 << 29, 1 << 30)
        out.append((6 * k + 1) * (12 * k + 1) * (18 * k + 1) % (1 << 64))
        k2 = rng.randrange(1 << 30, 1 << 31)
        out.append((k2 + 1) * (2 * k2 + 1))
    return out


SINGLE_PRIMES = [
    # p, b, c, N0, N1, mod, res  -- orders of b mod p far below the BSGS step count
    ((1 << 61) - 1, 2, -1, 0, 10_000_000, 1, 0),        # ord 61: b^n == 1 for n == 0 mod 61
    ((1 << 61) - 1, 2, -8, 5, 10_000, 1, 0),
    ((1 << 61) - 1, 2, -3, 0, 10_000_000, 1, 0),         # no solution
    ((1 << 61) - 1, 2, 1, 0, 1_000_000, 2, 1),
    ((1 << 31) - 1, 2, -4, 10, 5_000_000, 3, 2),
    ((1 << 31) - 1, 8, -64, 0, 1_000_000, 1, 0),
    (1_111_111_111_111_111_111, 10, -1, 0, 10_000_000, 1, 0),   # R19, ord(10) = 19
    (1_111_111_111_111_111_111, 10, -1000, 7, 2_000_000, 6, 3),
    (1_111_111_111_111_111_111, 10, 1, 0, 10_000_000, 1, 0),
    (65_537, 2, -1, 0, 100_000, 1, 0),                    # ord 32
    (65_537, 2, 1, 3, 100_000, 2, 0),
    (65_537, 3, 5, 0, 1_000_000, 1, 0),
    (999_999_000_001, 10, -1, 0, 10_000_000, 6, 0),      # divides 10^12 - 1... order 12
    (4_611_686_018_427_387_847, 2, -25, 0, 10_000_000, 1, 0),  # largest prime below 2^62
    (4_611_686_018_427_387_847, 3, 17, 100, 5_000_000, 12, 4),
]


def main():
    if not Reference.available():
        sys.exit("oracle/_ref/libmps_ref.so is missing: run `make -C oracle ref` where the reference is mounted")
    ref = Reference()
    t0 = time.time()

    # the small CPU-runnable config, full
    it = make_item(2, -25, 10**6, 10**8, 0, 100_000, 2, 1)
    rels, nprimes = ref.relations(10**6, 10**8, it)
    text = relation_lines(rels)
    with gzip.GzipFile(os.path.join(OUT, "c1_relations.txt.gz"), "wb", mtime=0) as f:
        f.write(text.encode())
    c1 = {"item": [2, -25, 10**6, 10**8, 0, 100_000, 2, 1], "primes": nprimes, "relations": len(rels),
          "md5": hashlib.md5(text.encode()).hexdigest()}
    print(f"c1: {nprimes} primes, {len(rels)} relations, md5 {c1['md5']} ({time.time() - t0:.1f}s)")

    cases = []
    for name, b, c, P0, P1, N0, N1, mod, res in ITEMS + c4_items(24, SEED, 300_000):
        t1 = time.time()
        it = make_item(b, c, P0, P1, N0, N1, mod, res)
        rels, nprimes = ref.relations(P0, P1, it)
        cases.append({"name": name, "item": [b, c, P0, P1, N0, N1, mod, res], "primes": nprimes,
                      "relations": [list(r) for r in rels]})
        print(f"{name}: {nprimes} primes, {len(rels)} relations ({time.time() - t1:.1f}s)")

    with open(os.path.join(OUT, "relations.json"), "w") as f:
        json.dump({"seed": SEED, "c1": c1, "cases": cases}, f, indent=0)
        f.write("\n")

    nums = sorted(set(IS_PRIME_CASES + strong_pseudoprimes_base2(200_000) + carmichael_like(40, SEED)))
    rng = random.Random(SEED)
    nums += [rng.randrange(3, 1 << 62) | 1 for _ in range(200)]
    with open(os.path.join(OUT, "is_prime.json"), "w") as f:
        json.dump([[n, int(ref.is_prime(n))] for n in nums], f)
        f.write("\n")

    singles = []
    for p, b, c, N0, N1, mod, res in SINGLE_PRIMES:
        assert ref.is_prime(p), p
        it = make_item(b, c, p, p + 1, N0, N1, mod, res)
        r = ref.run_bsgs(p, it)
        singles.append({"p": p, "item": [b, c, p, p + 1, N0, N1, mod, res], "relation": list(r) if r else None,
                        "order": ref.mult_order(b % p, p)})
    with open(os.path.join(OUT, "single_primes.json"), "w") as f:
        json.dump(singles, f, indent=0)
        f.write("\n")
    print(f"done in {time.time() - t0:.1f}s")


if __name__ == "__main__":
    main()
