"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
from __future__ import annotations

import gzip
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "libmps_oracle.so")
    src = os.path.join(ROOT, "oracle", "mps_oracle.c")
    if not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


@pytest.fixture(scope="session")
def oracle():
    _ensure_oracle()
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "relations.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_c1_lines():
    with gzip.open(os.path.join(GOLDEN, "c1_relations.txt.gz"), "rt") as f:
        return f.read()


@pytest.fixture(scope="session")
def golden_is_prime():
    with open(os.path.join(GOLDEN, "is_prime.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_single_primes():
    with open(os.path.join(GOLDEN, "single_primes.json")) as f:
        return json.load(f)
