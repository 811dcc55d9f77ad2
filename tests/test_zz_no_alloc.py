"""mps_chunk_relations_noalloc: the entry point for callers that cannot
allocate device memory where they sieve (their memory is owned by another
framework's pool, or cudaMalloc's device-wide synchronisation is not allowed
in their loop).  It keeps all scratch in one static device array, so its
results must equal the regular entry point's, call after call.

This file is collected last on purpose: if it fails, every other test has
already run.  It must pass in a fresh process (where its first call sets the
scratch up) as well as after the rest of the suite.
"""
from __future__ import annotations

import ctypes

import pytest

pytestmark = pytest.mark.gpu

SPAN_LIMIT = 1 << 19


def _noalloc(mps_lib):
    lib = mps_lib.load_library()
    fn = lib.mps_chunk_relations_noalloc
    fn.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(mps_lib.Item), ctypes.POINTER(mps_lib.Relation),
                   ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    fn.restype = ctypes.c_int

    def call(lo, hi, item, cap=1 << 16):
        buf = (mps_lib.Relation * cap)()
        n = ctypes.c_size_t()
        rc = fn(lo, hi, ctypes.byref(item), buf, cap, ctypes.byref(n))
        return rc, [(buf[i].p, buf[i].M, buf[i].q) for i in range(min(n.value, cap))], n.value

    return call


CASES = [
    # b, c, lo, hi, N0, N1, mod, res
    (2, -25, 10_000_000_000, 10_000_000_000 + SPAN_LIMIT, 3_600_000, 5_000_000, 2, 1),
    (10, 111, 10**12, 10**12 + SPAN_LIMIT, 0, 10_000_000, 6, 4),
    (2, -25, 2, 300_000, 0, 1_000, 1, 0),                        # small primes, p = 2
    ((1 << 80) + 3, -1, 10**9, 10**9 + SPAN_LIMIT, 0, 50_000, 2, 0),   # a relation for every prime: splits
]


def test_matches_regular_entry_point_twice(siever, mps_lib):
    call = _noalloc(mps_lib)
    for b, c, lo, hi, N0, N1, mod, res in CASES:
        item = mps_lib.make_item(b, c, lo, hi, N0, N1, mod, res)
        want = siever.chunk_relations(lo, hi, item)
        for _ in range(2):                                   # two calls in a row share the scratch
            rc, got, n = call(lo, hi, item)
            assert rc == mps_lib.MPS_OK
            assert n == len(want)
            assert got == want, (b, c, lo, hi)


def test_matches_golden_relations(mps_lib, golden):
    """Slices of non-empty reference-built golden items, each no wider than
    the entry point takes, against the golden relations of that slice."""
    call = _noalloc(mps_lib)
    for name in ("c2_low", "c3_low", "small_p_2", "selftest"):
        case = next(c for c in golden["cases"] if c["name"] == name)
        b, c, P0, P1, N0, N1, mod, res = case["item"]
        hi = min(P1, P0 + SPAN_LIMIT)
        want = [tuple(r) for r in case["relations"] if r[0] < hi]
        item = mps_lib.make_item(b, c, P0, hi, N0, N1, mod, res)
        for _ in range(2):
            rc, got, n = call(P0, hi, item)
            assert rc == mps_lib.MPS_OK and n == len(want)
            assert got == want, name


def test_rejects_ranges_beyond_its_scratch(mps_lib):
    call = _noalloc(mps_lib)
    item = mps_lib.make_item(2, -25, 10**9, 10**9 + SPAN_LIMIT + 2, 0, 1000, 1, 0)
    rc, _, _ = call(10**9, 10**9 + SPAN_LIMIT + 2, item)
    assert rc == mps_lib.MPS_E_RANGE
    # and still answers afterwards
    rc, got, _ = call(10**9, 10**9 + 1000, item)
    assert rc == mps_lib.MPS_OK
