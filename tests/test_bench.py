"""bench.py's own arithmetic, on CPU: the sieve's algorithmic work per odd
number, the CPU baseline's chunking (every host thread busy to the end of the
sample), the tuning summary, and the relations.p text it checks parity with."""
from __future__ import annotations

import math

import bench


def test_sieve_marks_per_odd():
    full = bench.sieve_marks_per_odd(10**13)             # every odd prime 3..65521 sieves
    assert abs(full - 2.1678) < 2e-3
    assert bench.sieve_marks_per_odd(10**6) < full       # only primes up to 1000
    want = sum(1.0 / q for q in range(3, 1000, 2) if all(q % d for d in range(3, math.isqrt(q) + 1, 2)))
    assert abs(bench.sieve_marks_per_odd(1000 * 1000) - want) < 1e-9


def test_cpu_chunking_keeps_every_thread_busy(monkeypatch):
    seen = {}

    class FakeRef:
        @staticmethod
        def available():
            return True

        def relations(self, lo, hi, it, threads, chunk):
            seen.update(width=hi - lo, threads=threads, chunk=chunk)
            return [], 1000

    import oracle.oracle as oo
    monkeypatch.setattr(oo, "Reference", FakeRef)
    for threads in (1, 8, 16, 64, 192):
        r = bench.cpu_reference_rate(bench.WORKLOADS["c2"], 100_000_000, threads)
        assert seen["chunk"] % (1 << 20) == 0 and seen["chunk"] >= 1 << 20
        chunks = -(-seen["width"] // seen["chunk"])
        assert r["busy_threads"] == min(threads, chunks)
        assert chunks >= min(threads, 95)                  # 1e8 holds 95 chunks of 2^20


def test_tuning_summary():
    reps = [dict(table_kind=2, load_shift=2, chains=2, warps=4, seg_words=2048, lanes=32, best_ns_per_prime=1.0,
                 default_ns_per_prime=1.5),
            dict(table_kind=2, load_shift=2, chains=2, warps=4, seg_words=2048, lanes=32, best_ns_per_prime=2.0,
                 default_ns_per_prime=2.0),
            dict(table_kind=0, load_shift=2, chains=4, warps=8, seg_words=4096, lanes=32, table_fill=192,
                 baby_scale=224, best_ns_per_prime=1.0, default_ns_per_prime=1.2)]
    s = bench.tuning_summary(reps, 3.0)
    assert s["classes"] == 3 and s["choices"] == {"kind2/load2^-2/lanes32/ch2/w4/seg2048": 2,
                                                      "kind0/fill192/scale224/ch4/w8/seg4096": 1}
    assert s["bsgs_gain_vs_default"]["max"] == 1.5 and s["bsgs_gain_vs_default"]["min"] == 1.0
    assert bench.tuning_summary([], 0.0)["bsgs_gain_vs_default"] is None


def test_relation_text():
    assert bench.relation_text([(7, 5, 3), (23, 1, 11)]) == "7, 5, 3\n23, 1, 11\n"
