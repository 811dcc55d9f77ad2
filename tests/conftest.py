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
PKG = os.path.join(ROOT, "mass-prime-siever_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "libmps_oracle.so")
    src = os.path.join(ROOT, "oracle", "mps_oracle.c")
    if not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


def _ensure_library():
    lib = os.path.join(PKG, "libmps_b200.so")
    srcs = [os.path.join(PKG, "csrc", f) for f in os.listdir(os.path.join(PKG, "csrc"))]
    srcs.append(os.path.join(ROOT, "include", "mps_gpu.h"))
    if not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(f) for f in srcs):
        subprocess.run(["make", "-s", "-C", PKG], check=True)
    return lib


@pytest.fixture(scope="session")
def mps_lib():
    _ensure_library()
    import mps_b200
    return mps_b200


@pytest.fixture(scope="session")
def siever(mps_lib):
    """One device context for the GPU tests (default tuning)."""
    s = mps_lib.Siever(0)
    yield s
    s.close()


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
