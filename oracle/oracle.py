"""ctypes bindings of the checker libraries (test infrastructure only).

`Oracle` wraps oracle/libmps_oracle.so, the C restatement of the reference's
hot path; `Reference` wraps oracle/_ref/libmps_ref.so, the reference's own
Math.hpp/Sieve.hpp compiled by oracle/Makefile.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU baseline use this module; the
product never does.
"""
from __future__ import annotations

import ctypes
import os
from typing import Iterable

HERE = os.path.dirname(os.path.abspath(__file__))
U64_MASK = (1 << 64) - 1


class Item(ctypes.Structure):
    """Factor=b,c,P0,P1,N0,N1[,mod,res]; b and c are signed 128-bit (hi:lo)."""

    _fields_ = [
        ("b_hi", ctypes.c_int64), ("b_lo", ctypes.c_uint64),
        ("c_hi", ctypes.c_int64), ("c_lo", ctypes.c_uint64),
        ("P0", ctypes.c_uint64), ("P1", ctypes.c_uint64),
        ("N0", ctypes.c_int64), ("N1", ctypes.c_int64),
        ("mod", ctypes.c_uint64), ("res", ctypes.c_uint64),
    ]


class Relation(ctypes.Structure):
    _fields_ = [("p", ctypes.c_uint64), ("M", ctypes.c_uint64), ("q", ctypes.c_uint64)]


class Counts(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("odds", "primes", "mr_mmul", "prep_mmul", "bsgs_mmul", "bsgs_primes", "relations")]


def split128(v: int) -> tuple[int, int]:
    """Signed 128-bit integer -> (signed high word, unsigned low word)."""
    if not -(1 << 127) <= v < (1 << 127):
        raise ValueError("value does not fit in a signed 128-bit integer")
    u = v & ((1 << 128) - 1)
    hi = u >> 64
    if hi >= 1 << 63:
        hi -= 1 << 64
    return hi, u & U64_MASK


def make_item(b: int, c: int, P0: int, P1: int, N0: int, N1: int, mod: int = 1, res: int = 0) -> Item:
    bh, bl = split128(b)
    ch, cl = split128(c)
    return Item(bh, bl, ch, cl, P0, P1, N0, N1, mod, res)


def _rel_list(buf, n) -> list[tuple[int, int, int]]:
    return [(buf[i].p, buf[i].M, buf[i].q) for i in range(n)]


class Oracle:
    """The C restatement (oracle/mps_oracle.c)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "libmps_oracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run `make -C oracle`)")
        L = self.lib = ctypes.CDLL(path)
        u64, sz, P = ctypes.c_uint64, ctypes.c_size_t, ctypes.POINTER
        L.mpo_is_prime64.argtypes = [u64]
        L.mpo_jacobi.argtypes = [u64, u64]
        L.mpo_mont_consts.argtypes = [u64, P(u64), P(u64), P(u64)]
        L.mpo_mont_mul.argtypes = [u64, u64, u64, u64]
        L.mpo_mont_mul.restype = u64
        L.mpo_powmod.argtypes = [u64, u64, u64]
        L.mpo_powmod.restype = u64
        L.mpo_sieve.argtypes = [u64, u64, P(u64), sz]
        L.mpo_sieve.restype = sz
        L.mpo_sieve_survivors.argtypes = [u64, u64, P(u64), sz]
        L.mpo_sieve_survivors.restype = sz
        L.mpo_mult_order.argtypes = [u64, u64]
        L.mpo_mult_order.restype = u64
        L.mpo_run_bsgs.argtypes = [u64, P(Item), P(Relation)]
        L.mpo_bsgs_smallest_j.argtypes = [u64, u64, u64, u64, u64]
        L.mpo_bsgs_smallest_j.restype = u64
        L.mpo_chunk_relations.argtypes = [u64, u64, P(Item), P(Relation), sz]
        L.mpo_chunk_relations.restype = sz
        L.mpo_chunk_relations_counted.argtypes = [u64, u64, P(Item), P(Relation), sz, P(Counts)]
        L.mpo_chunk_relations_counted.restype = sz
        L.mpo_relations_threaded.argtypes = [u64, u64, P(Item), P(Relation), sz, ctypes.c_int, u64]
        L.mpo_relations_threaded.restype = sz

    def is_prime(self, n: int) -> bool:
        return bool(self.lib.mpo_is_prime64(n))

    def jacobi(self, a: int, n: int) -> int:
        return self.lib.mpo_jacobi(a, n)

    def mont_consts(self, n: int) -> tuple[int, int, int]:
        a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self.lib.mpo_mont_consts(n, a, b, c)
        return a.value, b.value, c.value

    def mult_order(self, b: int, p: int) -> int:
        return self.lib.mpo_mult_order(b, p)

    def _vec(self, fn, lo, hi, cap):
        buf = (ctypes.c_uint64 * max(cap, 1))()
        n = fn(lo, hi, buf, cap)
        if n > cap:
            return self._vec(fn, lo, hi, n)
        return list(buf[:n])

    def primes(self, lo: int, hi: int, cap: int = 1 << 16) -> list[int]:
        return self._vec(self.lib.mpo_sieve, lo, hi, cap)

    def survivors(self, lo: int, hi: int, cap: int = 1 << 16) -> list[int]:
        return self._vec(self.lib.mpo_sieve_survivors, lo, hi, cap)

    def run_bsgs(self, p: int, item: Item):
        r = Relation()
        return (r.p, r.M, r.q) if self.lib.mpo_run_bsgs(p, ctypes.byref(item), ctypes.byref(r)) else None

    def bsgs_smallest_j(self, p: int, B: int, G0: int, t: int, jcount: int):
        j = self.lib.mpo_bsgs_smallest_j(p, B, G0, t, jcount)
        return None if j == U64_MASK else j

    def chunk_relations(self, lo: int, hi: int, item: Item, cap: int = 1 << 16):
        buf = (Relation * cap)()
        n = self.lib.mpo_chunk_relations(lo, hi, ctypes.byref(item), buf, cap)
        if n > cap:
            return self.chunk_relations(lo, hi, item, n)
        return _rel_list(buf, n)

    def chunk_counts(self, lo: int, hi: int, item: Item, cap: int = 1 << 16):
        buf = (Relation * cap)()
        c = Counts()
        n = self.lib.mpo_chunk_relations_counted(lo, hi, ctypes.byref(item), buf, cap, ctypes.byref(c))
        return _rel_list(buf, min(n, cap)), {k: getattr(c, k) for k, _ in Counts._fields_}

    def relations(self, lo: int, hi: int, item: Item, threads: int = 0, chunk: int = 1 << 24,
                  cap: int = 1 << 20):
        threads = threads or os.cpu_count() or 1
        buf = (Relation * cap)()
        n = self.lib.mpo_relations_threaded(lo, hi, ctypes.byref(item), buf, cap, threads, chunk)
        if n > cap:
            return self.relations(lo, hi, item, threads, chunk, n)
        return _rel_list(buf, n)


class Reference:
    """The reference's own Math.hpp/Sieve.hpp (oracle/_ref/libmps_ref.so)."""

    PATH = os.path.join(HERE, "_ref", "libmps_ref.so")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.PATH)

    def __init__(self, path: str | None = None):
        path = path or self.PATH
        L = self.lib = ctypes.CDLL(path)
        u64, sz, P = ctypes.c_uint64, ctypes.c_size_t, ctypes.POINTER
        L.ref_is_prime64.argtypes = [u64]
        L.ref_run_bsgs.argtypes = [u64, P(Item), P(Relation)]
        L.ref_mult_order.argtypes = [u64, u64]
        L.ref_mult_order.restype = u64
        L.ref_sieve.argtypes = [u64, u64, P(u64), sz]
        L.ref_sieve.restype = sz
        L.ref_chunk_relations.argtypes = [u64, u64, P(Item), P(Relation), sz, P(u64)]
        L.ref_chunk_relations.restype = sz
        L.ref_relations_threaded.argtypes = [u64, u64, P(Item), P(Relation), sz, ctypes.c_int, u64, P(u64)]
        L.ref_relations_threaded.restype = sz

    def is_prime(self, n: int) -> bool:
        return bool(self.lib.ref_is_prime64(n))

    def run_bsgs(self, p: int, item: Item):
        r = Relation()
        return (r.p, r.M, r.q) if self.lib.ref_run_bsgs(p, ctypes.byref(item), ctypes.byref(r)) else None

    def mult_order(self, b: int, p: int) -> int:
        return self.lib.ref_mult_order(b, p)

    def relations(self, lo: int, hi: int, item: Item, threads: int = 0, chunk: int = 1 << 24,
                  cap: int = 1 << 20):
        threads = threads or os.cpu_count() or 1
        buf = (Relation * cap)()
        np_ = ctypes.c_uint64()
        n = self.lib.ref_relations_threaded(lo, hi, ctypes.byref(item), buf, cap, threads, chunk,
                                            ctypes.byref(np_))
        if n > cap:
            return self.relations(lo, hi, item, threads, chunk, n)
        return _rel_list(buf, n), np_.value


def relation_lines(rels: Iterable[tuple[int, int, int]]) -> str:
    """relations.p text in the reference's "%llu, %llu, %llu\\n" format (Worker.hpp:294-297)."""
    return "".join(f"{p}, {M}, {q}\n" for p, M, q in rels)
