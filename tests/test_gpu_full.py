"""Parity at the benchmark configurations' own sizes: the device path against
the reference-built fixtures of tests/golden/make_full_golden.py (the
reference's own segmented_sieve + run_bsgs over the whole range).

  C2  b=10 c=111, 10^12 <= p < 10^12 + 10^10, n in [0, 10^7), n == 4 mod 6:
      361,840,208 primes, 592 relations
  C3  b=2 c=-25, 9.5e13 <= p < 9.5e13 + 2e10, n in [3.6e6, 5e6), n == 1 mod 2:
      621,389,051 primes, 4 relations
  C4  the 64 mixed-batch items (seed 20261203), first 10^8 of each P range:
      245,224,609 primes, 5,709 relations
Integer work: every comparison is exact."""
from __future__ import annotations

import gzip
import hashlib
import json
import os

import pytest

from conftest import GOLDEN
from oracle.oracle import relation_lines

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def full():
    with open(os.path.join(GOLDEN, "full.json")) as f:
        return json.load(f)


def _lines(name):
    with gzip.open(os.path.join(GOLDEN, f"{name}_full.txt.gz"), "rt") as f:
        return f.read()


@pytest.mark.parametrize("name", ["c2", "c3"])
def test_full_config_relations(siever, mps_lib, full, name):
    g = full[name]
    got = siever.item_relations(mps_lib.make_item(*g["item"]))
    text = relation_lines(got)
    assert len(got) == g["relations"]
    assert hashlib.md5(text.encode()).hexdigest() == g["md5"]
    assert text == _lines(name)


@pytest.mark.parametrize("name", ["c2", "c3"])
def test_full_config_prime_count(siever, full, name):
    g = full[name]
    assert siever.count_primes(g["item"][2], g["item"][3]) == g["primes"]


def test_c4_first_1e8_batched_and_alone(siever, mps_lib):
    with open(os.path.join(GOLDEN, "c4_1e8.json")) as f:
        g = json.load(f)
    import workloads
    specs = workloads.c4_items(max_width=g["prefix"])
    assert [list(s) for s in specs] == [c["item"] for c in g["cases"]]
    items = [mps_lib.make_item(*s) for s in specs]
    got = siever.batch_relations(items)
    for k, case in enumerate(g["cases"]):
        assert [[p, M, q] for i, p, M, q in got if i == k] == case["relations"], case["name"]
    for k in (5, 20, 43):                                  # the densest items, alone
        assert [list(r) for r in siever.item_relations(items[k])] == g["cases"][k]["relations"]


def test_c2_plain_method_path(mps_lib, full):
    """The plain per-item comparator of the bench (the reference's plain-method
    filter, stage-by-stage launches) gives the same C2 relations."""
    g = full["c2"]
    with mps_lib.Siever(0, plain=1, class_modulus=1) as s:
        got = s.item_relations(mps_lib.make_item(*g["item"]))
    assert hashlib.md5(relation_lines(got).encode()).hexdigest() == g["md5"]
