"""The benchmark workloads (synthetic, seeded): the five configurations.

  c1  small CPU-runnable: b=2 c=-25, 10^6 <= p < 10^8, 0 <= n < 10^5, n == 1 (mod 2)
  c2  plain GPU path, full size: b=10 c=111, 10^12 <= p < 10^12 + 10^10, 0 <= n < 10^7, n == 4 (mod 6)
  c3  residue classes: b=2 c=-25, 9.5e13 <= p < 9.5e13 + 2e10, 3.6e6 <= n < 5e6, n == 1 (mod 2)
  c4  64 mixed items drawn from a fixed seed (below)
  c5  items drawn as in c4 arriving by a seeded Poisson process (the serving stream)

No public dataset is involved; every input is generated here.
"""
from __future__ import annotations

import math
import random

C4_SEED = 20261203

SINGLE = {
    "c1": (2, -25, 10**6, 10**8, 0, 100_000, 2, 1),
    "c2": (10, 111, 10**12, 10**12 + 10**10, 0, 10**7, 6, 4),
    "c3": (2, -25, 95 * 10**12, 95 * 10**12 + 2 * 10**10, 3_600_000, 5_000_000, 2, 1),
}


def draw_item(rng: random.Random) -> tuple:
    """One item with the mixed-batch distributions:
    b uniform in {2,3,5,6,7,10,12}; c uniform over the nonzero integers of
    [-999, 999] with gcd(b, c) = 1 (redrawn); P0 = floor(10^U(9,14));
    P width = floor(10^U(8,10)); N0 uniform in [0, 10^6]; N width =
    floor(10^U(4,7)); mod uniform in {1,2,6,12}; res uniform in [0, mod)."""
    b = rng.choice([2, 3, 5, 6, 7, 10, 12])
    while True:
        c = rng.randint(-999, 999)
        if c != 0 and math.gcd(b, abs(c)) == 1:
            break
    P0 = int(10 ** rng.uniform(9, 14))
    width = int(10 ** rng.uniform(8, 10))
    N0 = rng.randint(0, 10**6)
    nw = int(10 ** rng.uniform(4, 7))
    mod = rng.choice([1, 2, 6, 12])
    res = rng.randrange(mod)
    return (b, c, P0, P0 + width, N0, N0 + nw, mod, res)


def c4_items(n: int = 64, seed: int = C4_SEED, max_width: int | None = None) -> list[tuple]:
    """The mixed batch; max_width caps each item's P width (the first
    max_width of every item) for quick runs."""
    rng = random.Random(seed)
    items = [draw_item(rng) for _ in range(n)]
    if max_width is not None:
        items = [(b, c, P0, min(P1, P0 + max_width), N0, N1, mod, res) for b, c, P0, P1, N0, N1, mod, res in items]
    return items


def c5_arrivals(rate_items_per_s: float, duration_s: float, seed: int = C4_SEED + 5,
                max_width: int | None = None) -> list[tuple[float, tuple]]:
    """(arrival time, item) pairs: a Poisson process of the given rate over
    duration_s, items drawn as in c4."""
    rng = random.Random(seed)
    t = 0.0
    out = []
    while True:
        t += rng.expovariate(rate_items_per_s)
        if t >= duration_s:
            break
        it = draw_item(rng)
        if max_width is not None:
            b, c, P0, P1, N0, N1, mod, res = it
            it = (b, c, P0, min(P1, P0 + max_width), N0, N1, mod, res)
        out.append((t, it))
    return out


def approx_primes(P0: int, P1: int) -> float:
    """li(P1) - li(P0) approximation of the prime count (for planning only)."""
    def li(x):
        lx = math.log(x)
        return x / lx * (1 + 1 / lx + 2 / lx**2 + 6 / lx**3)
    return li(P1) - li(P0)
