"""The C restatement (oracle/) against the fixtures made by the reference itself.

These pin the oracle before any GPU result is compared with it.
"""
from __future__ import annotations

import hashlib
import math
import random

import pytest

from oracle.oracle import make_item, relation_lines


def test_is_prime_golden(oracle, golden_is_prime):
    bad = [(n, v) for n, v in golden_is_prime if oracle.is_prime(n) != bool(v)]
    assert not bad, bad[:5]


def test_jacobi_matches_euler(oracle):
    rng = random.Random(5)
    for p in [1009, 65521, 1_000_000_007, (1 << 61) - 1, 4_611_686_018_427_387_847]:
        for _ in range(50):
            a = rng.randrange(1, p)
            e = pow(a, (p - 1) // 2, p)
            assert oracle.jacobi(a, p) == (1 if e == 1 else -1)
    # composite moduli: multiplicativity in the denominator
    for _ in range(200):
        m, n = rng.randrange(3, 10**6) | 1, rng.randrange(3, 10**6) | 1
        a = rng.randrange(0, 10**9)
        assert oracle.jacobi(a, m * n) == oracle.jacobi(a, m) * oracle.jacobi(a, n)


def test_montgomery_constants(oracle):
    rng = random.Random(7)
    for _ in range(200):
        n = rng.randrange(3, 1 << 62) | 1
        ninv, one, r2 = oracle.mont_consts(n)
        assert (n * ninv) % (1 << 64) == (1 << 64) - 1
        assert one == (1 << 64) % n and r2 == (1 << 128) % n


def test_sieve_counts(oracle):
    assert oracle.primes(0, 100) == [p for p in range(100) if p > 1 and all(p % q for q in range(2, p))]
    assert len(oracle.primes(10**6, 2 * 10**6, 1 << 17)) == 70435
    # above 65536^2 the survivors of the sieve by 3..65521 include composites
    lo = 10**12
    surv = oracle.survivors(lo, lo + 100_000)
    primes = oracle.primes(lo, lo + 100_000)
    assert set(primes) <= set(surv) and len(primes) == 3614
    assert all(all(v % q for q in (3, 5, 7, 11, 13, 65521)) for v in surv)


def test_single_primes_golden(oracle, golden_single_primes):
    for case in golden_single_primes:
        p = case["p"]
        it = make_item(*case["item"])
        got = oracle.run_bsgs(p, it)
        want = tuple(case["relation"]) if case["relation"] else None
        assert got == want, case
        assert oracle.mult_order(case["item"][0] % p, p) == case["order"]


def test_bsgs_smallest_j_bruteforce(oracle):
    rng = random.Random(11)
    for _ in range(300):
        p = rng.choice([1009, 7919, 65537, 104729, 1_000_003])
        B = rng.randrange(1, p)
        if rng.random() < 0.2:
            B = pow(rng.randrange(2, p), (p - 1) // rng.choice([2, 4, 8, 16]), p) or 1
        G0 = rng.randrange(1, p)
        jcount = rng.randrange(1, 3000)
        t = G0 * pow(B, rng.randrange(0, 4000), p) % p if rng.random() < 0.7 else rng.randrange(1, p)
        want = None
        v = G0
        for j in range(jcount):
            if v == t:
                want = j
                break
            v = v * B % p
        assert oracle.bsgs_smallest_j(p, B, G0, t, jcount) == want


@pytest.mark.parametrize("name", ["selftest", "c2_low", "c3_low", "b12_mod12", "small_p_2", "small_p_10",
                                  "small_p_negb", "p_div_b_and_c", "p_div_b_only", "p_div_c_only",
                                  "c_128bit", "b_128bit", "narrow_n", "empty_class", "mod_gt_span",
                                  "mod3", "mod48"])
def test_relations_golden(oracle, golden, name):
    case = next(c for c in golden["cases"] if c["name"] == name)
    b, c, P0, P1, N0, N1, mod, res = case["item"]
    got = oracle.relations(P0, P1, make_item(b, c, P0, P1, N0, N1, mod, res))
    assert [list(r) for r in got] == case["relations"]


def test_relations_golden_c4(oracle, golden):
    for case in golden["cases"]:
        if not case["name"].startswith("c4_"):
            continue
        b, c, P0, P1, N0, N1, mod, res = case["item"]
        got = oracle.relations(P0, P1, make_item(b, c, P0, P1, N0, N1, mod, res))
        assert [list(r) for r in got] == case["relations"], case["name"]


@pytest.mark.slow
def test_c1_full_md5(oracle, golden):
    """The whole small CPU-runnable config: 5,682,957 primes, 14,090 relations."""
    c1 = golden["c1"]
    b, c, P0, P1, N0, N1, mod, res = c1["item"]
    got = oracle.relations(P0, P1, make_item(b, c, P0, P1, N0, N1, mod, res))
    text = relation_lines(got)
    assert len(got) == c1["relations"]
    assert hashlib.md5(text.encode()).hexdigest() == c1["md5"]


def test_counts_consistent(oracle):
    it = make_item(10, 111, 10**12, 10**12 + 10**6, 0, 10**7, 6, 4)
    rels, cnt = oracle.chunk_counts(10**12, 10**12 + 10**6, it)
    assert cnt["odds"] == 500_000
    assert cnt["primes"] == len(oracle.primes(10**12, 10**12 + 10**6, 1 << 16))
    # every prime pays ~12 strong tests of ~log2 p squarings
    assert cnt["mr_mmul"] > 12 * 39 * cnt["primes"]
    assert 0 < cnt["bsgs_primes"] < cnt["primes"]
    m = math.isqrt(10**7 // 6) + 1
    assert cnt["bsgs_mmul"] <= cnt["bsgs_primes"] * 2 * (m + 2)


def test_mult_order_when_p_minus_1_has_two_large_factors(oracle):
    """p - 1 = m q1 q2 with q1, q2 primes above 65521: the order needs the
    cofactor split (rho on the device).  The oracle's order is the true order."""
    sympy = pytest.importorskip("sympy")
    for p in (32505883140163, 15332064649691, 41010969574327, 119026820723087, 664006356569749, 79226575236629):
        for b in (2, 3, 10, 12):
            assert oracle.mult_order(b, p) == sympy.n_order(b, p), (b, p)
