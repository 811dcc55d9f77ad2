"""Parity of the sm_100a kernels with the oracle (CPU restatement of the
reference), through the C-ABI.  Integer work: every comparison is exact."""
from __future__ import annotations

import hashlib
import random

import pytest

from oracle.oracle import make_item as oracle_item, relation_lines

pytestmark = pytest.mark.gpu


def item(mps_lib, spec):
    b, c, P0, P1, N0, N1, mod, res = spec
    return mps_lib.make_item(b, c, P0, P1, N0, N1, mod, res)


# ---------------------------------------------------------------- kernels --

@pytest.mark.parametrize("lo,hi", [
    (0, 200_000), (3, 4096), (999_000, 1_131_072), (65521 * 65521 - 300_000, 65521 * 65521 + 300_000),
    (10**12, 10**12 + 400_000), (95 * 10**12 + 1, 95 * 10**12 + 262_145), ((1 << 62) - 500_000, 1 << 62),
    (1_000_003, 1_000_004), (1_000_004, 1_000_005),
])
def test_survivors_match_oracle(siever, oracle, lo, hi):
    want = oracle.survivors(lo, hi)
    got = siever.survivors(lo, hi)
    assert got == want


def test_is_prime_golden(siever, golden_is_prime):
    nums = [n for n, _ in golden_is_prime if n < (1 << 62)]
    want = [v for n, v in golden_is_prime if n < (1 << 62)]
    assert siever.is_prime(nums) == want


def test_is_prime_random(siever, oracle):
    rng = random.Random(3)
    nums = [rng.randrange(3, 1 << 62) | 1 for _ in range(5000)]
    nums += oracle.primes(10**12, 10**12 + 20_000)
    assert siever.is_prime(nums) == [int(oracle.is_prime(n)) for n in nums]


def _bsgs_cases(seed, count):
    rng = random.Random(seed)
    primes = [1009, 65537, 1_000_003, 999_999_000_001, (1 << 61) - 1, 4_611_686_018_427_387_847, 2_147_483_647]
    cases = []
    for _ in range(count):
        p = rng.choice(primes)
        kind = rng.random()
        if kind < 0.15:
            B = pow(rng.randrange(2, p), (p - 1) // rng.choice([2, 4, 8, 16, 32, 64]), p) or 1   # small order
        elif kind < 0.2:
            B = 1
        elif kind < 0.25:
            B = p - 1
        else:
            B = rng.randrange(2, p)
        G0 = rng.randrange(1, p)
        jcount = rng.choice([2, 3, 64, 65, 1000, 4097, rng.randrange(2, 200_000), 10_000_000])
        if rng.random() < 0.6:
            t = G0 * pow(B, rng.randrange(0, 2 * jcount), p) % p
        else:
            t = rng.randrange(1, p)
        cases.append((p, B, G0, t, jcount))
    return cases


@pytest.mark.parametrize("table_bits", [5, 6, 9, 12, 13])
@pytest.mark.parametrize("table_kind", [0, 1, 2, 3])
def test_bsgs_smallest_j(mps_lib, oracle, table_bits, table_kind):
    cases = _bsgs_cases(100 + table_bits, 400)
    with mps_lib.Siever(0, table_kind=table_kind) as s:
        got = s.bsgs(cases, table_bits=table_bits)
    want = [oracle.bsgs_smallest_j(*c) for c in cases]
    bad = [(c, g, w) for c, g, w in zip(cases, got, want) if g != w]
    assert not bad, bad[:3]


def test_order(siever, oracle):
    rng = random.Random(9)
    pairs = []
    # the last six: p - 1 = m q1 q2 with q1, q2 primes above 65521, so the cofactor is split by rho
    for p in (oracle.primes(10**6, 10**6 + 3000) + oracle.primes(10**12, 10**12 + 3000) +
              [(1 << 61) - 1, 4_611_686_018_427_387_847, 1_111_111_111_111_111_111, 999_999_000_001] +
              [32505883140163, 15332064649691, 41010969574327, 119026820723087, 664006356569749, 79226575236629]):
        pairs.append((rng.choice([2, 3, 5, 10, 12, 7]), p))
    want = [oracle.mult_order(b, p) for b, p in pairs]
    assert siever.order(pairs) == want


# -------------------------------------------------------------- relations --

def test_single_primes(siever, mps_lib, golden_single_primes):
    for case in golden_single_primes:
        p = case["p"]
        b, c, _, _, N0, N1, mod, res = case["item"]
        it = mps_lib.make_item(b, c, p, p + 1, N0, N1, mod, res)
        got = siever.chunk_relations(p, p + 1, it)
        want = [tuple(case["relation"])] if case["relation"] else []
        assert got == want, case


def test_golden_relations(siever, mps_lib, golden):
    for case in golden["cases"]:
        b, c, P0, P1, N0, N1, mod, res = case["item"]
        got = siever.item_relations(mps_lib.make_item(b, c, P0, P1, N0, N1, mod, res))
        assert [list(r) for r in got] == case["relations"], case["name"]


def test_c1_full(siever, mps_lib, golden):
    """The CPU-runnable config: 14,090 relations, md5 of the sorted relations.p."""
    c1 = golden["c1"]
    got = siever.item_relations(item(mps_lib, c1["item"]))
    assert len(got) == c1["relations"]
    assert hashlib.md5(relation_lines(got).encode()).hexdigest() == c1["md5"]


def test_c1_prime_count(siever, golden):
    assert siever.count_primes(10**6, 10**8) == golden["c1"]["primes"]


@pytest.mark.parametrize("tuning", [
    dict(plain=1), dict(full_mr=1), dict(table_bits=6), dict(table_bits=9, max_baby=100),
    dict(class_modulus=2), dict(class_modulus=48), dict(class_modulus=720), dict(chunk_odds=40_000),
    dict(bsgs_warps=1), dict(bsgs_warps=8, table_bits=11), dict(table_kind=1), dict(table_kind=1, chains=4),
    dict(chains=1), dict(chains=4), dict(table_bits=7, max_baby=256), dict(graphs_off=1),
    dict(table_kind=2), dict(table_kind=2, chains=1), dict(table_kind=2, chains=4), dict(table_kind=2, load_shift=3),
    dict(table_kind=2, load_shift=1, table_bits=7), dict(table_kind=2, bsgs_warps=8), dict(class_modulus=1),
    dict(class_modulus=1, plain=1), dict(table_kind=2, lanes=16), dict(table_kind=2, lanes=8, chains=1),
    dict(table_kind=2, lanes=8, bsgs_warps=8), dict(table_kind=2, lanes=16, load_shift=3, plain=1),
    dict(table_kind=3), dict(table_kind=3, chains=4), dict(table_kind=3, load_shift=3, chains=1),
    dict(table_kind=3, load_shift=3, bsgs_warps=8, plain=1),
])
def test_tunings_give_identical_relations(mps_lib, oracle, tuning):
    specs = [(2, -25, 10**10, 10**10 + 4_000_000, 3_600_000, 5_000_000, 2, 1),
             (10, 111, 10**9, 10**9 + 4_000_000, 0, 10_000_000, 6, 4),
             (7, -3, 5 * 10**9, 5 * 10**9 + 2_000_000, 0, 1_000_000, 1, 0),
             (3, 5, 2, 300_000, 0, 5_000, 12, 7)]
    with mps_lib.Siever(0, **tuning) as s:
        for spec in specs:
            got = s.item_relations(item(mps_lib, spec))
            want = oracle.relations(spec[2], spec[3], oracle_item(*spec))
            assert got == want, (tuning, spec)


def test_random_items_vs_oracle(siever, mps_lib, oracle):
    rng = random.Random(77)
    for _ in range(30):
        b = rng.choice([2, 3, 5, 6, 7, 10, 12, 13, -2, 1_000_003])
        c = rng.choice([x for x in range(-999, 1000) if x])
        P0 = int(10 ** rng.uniform(3, 13))
        P1 = P0 + rng.randrange(1, 300_000)
        N0 = rng.randrange(0, 10**6)
        N1 = N0 + int(10 ** rng.uniform(0, 6.5)) + 1
        mod = rng.choice([1, 2, 3, 4, 6, 12, 24, 30, 48, 100])
        res = rng.randrange(mod)
        spec = (b, c, P0, P1, N0, N1, mod, res)
        got = siever.item_relations(item(mps_lib, spec))
        want = oracle.relations(P0, P1, oracle_item(*spec))
        assert got == want, spec


# ----------------------------------------------------------------- compat --

def test_sieve_filter_compat(siever, mps_lib, oracle):
    spec = (2, -25, 10**10, 10**10 + 20_000_000, 3_600_000, 5_000_000, 2, 1)
    it = item(mps_lib, spec)
    flagged = siever.sieve_filter(spec[2], spec[3], it)
    want = oracle.relations(spec[2], spec[3], oracle_item(*spec))
    assert flagged == [r[0] for r in want]
    with pytest.raises(mps_lib.MpsError) as e:
        siever.sieve_filter(3, 1000, it)
    assert e.value.code == mps_lib.MPS_E_RANGE


def test_filter_compat(siever, mps_lib, oracle):
    spec = (10, 111, 10**9, 10**9 + 3_000_000, 0, 10_000_000, 6, 4)
    primes = oracle.primes(spec[2], spec[3], 1 << 18)
    flags = siever.filter(primes, item(mps_lib, spec))
    want = {r[0] for r in oracle.relations(spec[2], spec[3], oracle_item(*spec))}
    assert [p for p, f in zip(primes, flags) if f] == sorted(want)


def test_batch_matches_alone(siever, mps_lib, golden):
    cases = [c for c in golden["cases"] if c["name"].startswith("c4_")] + \
            [c for c in golden["cases"] if c["name"] in ("selftest", "c2_low", "small_p_2", "mod48")]
    items = [item(mps_lib, c["item"]) for c in cases]
    got = siever.batch_relations(items)
    for k, c in enumerate(cases):
        mine = [[p, M, q] for i, p, M, q in got if i == k]
        assert mine == c["relations"], c["name"]


# ----------------------------------------------------------------- errors --

def test_argument_errors(siever, mps_lib):
    bad = [
        ((2, -25, 10, 5, 0, 10, 1, 0), mps_lib.MPS_E_ARG),                 # P0 >= P1
        ((2, -25, 10, (1 << 62) + 2, 0, 10, 1, 0), mps_lib.MPS_E_RANGE),   # P1 > 2^62
        ((2, -25, 10, 100, 5, 5, 1, 0), mps_lib.MPS_E_ARG),                # N0 >= N1
        ((2, -25, 10, 100, 0, 10_000_001, 1, 0), mps_lib.MPS_E_RANGE),    # N span > 10^7
        ((2, -25, 10, 100, 0, 10, 6, 6), mps_lib.MPS_E_ARG),               # res >= mod
    ]
    for spec, code in bad:
        with pytest.raises(mps_lib.MpsError) as e:
            siever.item_relations(item(mps_lib, spec))
        assert e.value.code == code, spec
    # the context stays usable
    assert siever.item_relations(item(mps_lib, (2, -25, 10**6, 10**6 + 100_000, 0, 1000, 1, 0))) is not None


def test_prime_count_above_2_32(siever, oracle):
    for lo in (10**12, 95 * 10**12, (1 << 52) + 7, (1 << 61)):
        assert siever.count_primes(lo, lo + 300_000) == len(oracle.primes(lo, lo + 300_000, 1 << 16))
