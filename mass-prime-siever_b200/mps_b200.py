"""ctypes binding of libmps_b200.so (the C-ABI of include/mps_gpu.h).

Used by the tests, bench.py and __graft_entry__.py.  The product is the
shared library and the C++ host (host/); this module only calls the C-ABI.
It raises when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmps_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "mps_gpu.h")
U64_MAX = (1 << 64) - 1

MPS_OK, MPS_E_ARG, MPS_E_RANGE, MPS_E_CAPACITY, MPS_E_TIMEOUT, MPS_E_CUDA, MPS_E_NODEV, MPS_E_STATE = \
    0, -1, -2, -3, -4, -5, -6, -7
ERROR_NAMES = {MPS_E_ARG: "MPS_E_ARG", MPS_E_RANGE: "MPS_E_RANGE", MPS_E_CAPACITY: "MPS_E_CAPACITY",
               MPS_E_TIMEOUT: "MPS_E_TIMEOUT", MPS_E_CUDA: "MPS_E_CUDA", MPS_E_NODEV: "MPS_E_NODEV",
               MPS_E_STATE: "MPS_E_STATE"}


class MpsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


class Item(ctypes.Structure):
    _fields_ = [
        ("b_hi", ctypes.c_int64), ("b_lo", ctypes.c_uint64),
        ("c_hi", ctypes.c_int64), ("c_lo", ctypes.c_uint64),
        ("P0", ctypes.c_uint64), ("P1", ctypes.c_uint64),
        ("N0", ctypes.c_int64), ("N1", ctypes.c_int64),
        ("mod", ctypes.c_uint64), ("res", ctypes.c_uint64),
    ]


class Relation(ctypes.Structure):
    _fields_ = [("p", ctypes.c_uint64), ("M", ctypes.c_uint64), ("q", ctypes.c_uint64)]


class Tuning(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_uint32), ("table_bits", ctypes.c_uint32),
        ("chunk_odds", ctypes.c_uint64), ("max_baby", ctypes.c_uint32),
        ("bsgs_warps", ctypes.c_uint32), ("class_modulus", ctypes.c_uint32),
        ("full_mr", ctypes.c_uint32), ("plain", ctypes.c_uint32),
        ("chains", ctypes.c_uint32), ("graphs_off", ctypes.c_uint32), ("table_kind", ctypes.c_uint32),
        ("load_shift", ctypes.c_uint32), ("lanes", ctypes.c_uint32), ("table_fill", ctypes.c_uint32),
        ("baby_scale", ctypes.c_uint32),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("odds", ctypes.c_uint64), ("survivors", ctypes.c_uint64), ("entries", ctypes.c_uint64),
        ("relations", ctypes.c_uint64), ("chunks", ctypes.c_uint64), ("device_ms", ctypes.c_double),
        ("bsgs_ms", ctypes.c_double), ("bsgs_launches", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint64),
        ("bsgs_steps", ctypes.c_uint64), ("sieve_ms", ctypes.c_double), ("prep_ms", ctypes.c_double),
        ("order_ms", ctypes.c_double), ("bsgs_baby_steps", ctypes.c_uint64),
    ]


class ServeConfig(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("max_active", ctypes.c_uint32),
                ("mem_budget_bytes", ctypes.c_uint64), ("piece_odds", ctypes.c_uint64),
                ("reserved", ctypes.c_uint32 * 8)]


class ServeStatus(ctypes.Structure):
    _fields_ = [("ticket", ctypes.c_uint64), ("state", ctypes.c_int32), ("error", ctypes.c_int32),
                ("p_done", ctypes.c_uint64), ("relations", ctypes.c_uint64),
                ("latency_ms", ctypes.c_double), ("queue_ms", ctypes.c_double),
                ("reserved_bytes", ctypes.c_uint64), ("relations_on_device", ctypes.c_int32), ("pad", ctypes.c_int32)]


class TuneReport(ctypes.Structure):
    _fields_ = [("k_bits", ctypes.c_uint32), ("mod", ctypes.c_uint32), ("p_digits", ctypes.c_uint32),
                ("candidates", ctypes.c_uint32), ("table_kind", ctypes.c_uint32), ("load_shift", ctypes.c_uint32),
                ("chains", ctypes.c_uint32), ("warps", ctypes.c_uint32), ("seg_words", ctypes.c_uint32),
                ("lanes", ctypes.c_uint32), ("table_fill", ctypes.c_uint32), ("baby_scale", ctypes.c_uint32),
                ("best_ns_per_prime", ctypes.c_double),
                ("default_ns_per_prime", ctypes.c_double), ("sieve_best_ms", ctypes.c_double),
                ("sieve_default_ms", ctypes.c_double), ("calib_bsgs_primes", ctypes.c_uint64)]


def split128(v: int) -> tuple[int, int]:
    if not -(1 << 127) <= v < (1 << 127):
        raise ValueError("value does not fit in a signed 128-bit integer")
    u = v & ((1 << 128) - 1)
    hi = u >> 64
    if hi >= 1 << 63:
        hi -= 1 << 64
    return hi, u & U64_MAX


def make_item(b: int, c: int, P0: int, P1: int, N0: int, N1: int, mod: int = 1, res: int = 0) -> Item:
    bh, bl = split128(b)
    ch, cl = split128(c)
    return Item(bh, bl, ch, cl, P0, P1, N0, N1, mod, res)


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the in-tree shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built: run `make -C mass-prime-siever_b200` (or build())")
    L = ctypes.CDLL(path)
    u64, u32, sz, P = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_size_t, ctypes.POINTER
    vp = ctypes.c_void_p
    L.mps_tuning_default.argtypes = [P(Tuning)]
    L.mps_open.argtypes = [ctypes.c_int, P(Tuning), P(vp)]
    L.mps_close.argtypes = [vp]
    L.mps_last_error.argtypes = [vp]
    L.mps_last_error.restype = ctypes.c_char_p
    L.mps_get_stats.argtypes = [vp, P(Stats)]
    L.mps_chunk_relations.argtypes = [vp, u64, u64, P(Item), P(Relation), sz, P(sz)]
    L.mps_item_relations.argtypes = [vp, P(Item), P(Relation), sz, P(sz)]
    L.mps_sieve_filter.argtypes = [vp, u64, u64, P(Item), P(u64), sz, P(sz)]
    L.mps_filter.argtypes = [vp, P(u64), sz, P(Item), P(ctypes.c_uint8)]
    L.mps_batch_relations.argtypes = [vp, P(Item), sz, P(Relation), P(u32), sz, P(sz)]
    L.mps_count_primes.argtypes = [vp, u64, u64, P(u64)]
    L.mps_take_relations.argtypes = [vp, P(Relation), P(u32), sz, P(sz)]
    L.mps_serve_config_default.argtypes = [P(ServeConfig)]
    L.mps_serve_open.argtypes = [ctypes.c_int, P(Tuning), P(ServeConfig), P(vp)]
    L.mps_serve_submit.argtypes = [vp, P(Item), P(u64)]
    L.mps_serve_wait.argtypes = [vp, u64, ctypes.c_double, P(ServeStatus)]
    L.mps_serve_result.argtypes = [vp, u64, P(Relation), sz, P(sz)]
    L.mps_serve_release.argtypes = [vp, u64]
    L.mps_serve_checkpoint.argtypes = [vp, u64, P(u64), P(u64)]
    L.mps_serve_close.argtypes = [vp]
    L.mps_serve_pool.argtypes = [vp, P(u64), P(u64), P(u32), P(u32)]
    L.mps_measure_peaks.argtypes = [vp, P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_double)]
    L.mps_measure_smem_peak.argtypes = [vp, P(ctypes.c_double)]
    L.mps_autotune.argtypes = [vp, P(Item), sz, P(TuneReport), sz, P(sz)]
    L.mps_tune_save.argtypes = [vp, ctypes.c_char_p]
    L.mps_tune_load.argtypes = [vp, ctypes.c_char_p]
    L.mps_tune_clear.argtypes = [vp]
    L.mps_test_survivors.argtypes = [vp, u64, u64, P(u64), sz, P(sz)]
    L.mps_test_is_prime.argtypes = [vp, P(u64), sz, P(ctypes.c_uint8)]
    L.mps_test_bsgs.argtypes = [vp, P(u64), sz, u32, P(u64)]
    L.mps_test_order.argtypes = [vp, P(u64), sz, P(u64)]
    _lib = L
    return L


def header_symbols(path: str = HEADER) -> list[str]:
    """Function names declared in include/mps_gpu.h."""
    text = open(path).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*|void)\s+(mps_\w+)\s*\(", text, re.M)))


def default_tuning(**kw) -> Tuning:
    L = load_library()
    t = Tuning()
    L.mps_tuning_default(ctypes.byref(t))
    for k, v in kw.items():
        if not hasattr(t, k):
            raise AttributeError(k)
        setattr(t, k, v)
    return t


class Siever:
    """One device context (mps_ctx).  Mirrors GpuSiever (Gpu.hpp:1040-1074):
    sieve_filter / filter with the same contracts, plus the exact relation
    calls.  Not thread-safe; serialise calls per instance."""

    def __init__(self, device: int = 0, tuning: Tuning | None = None, **kw):
        self.lib = load_library()
        if tuning is None:
            tuning = default_tuning(**kw)
        self.ctx = ctypes.c_void_p()
        rc = self.lib.mps_open(device, ctypes.byref(tuning), ctypes.byref(self.ctx))
        if rc != MPS_OK:
            raise MpsError(rc, "mps_open failed (no CUDA device?)")

    def close(self):
        if self.ctx:
            self.lib.mps_close(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != MPS_OK:
            raise MpsError(rc, self.lib.mps_last_error(self.ctx).decode())

    def stats(self) -> dict:
        s = Stats()
        self._check(self.lib.mps_get_stats(self.ctx, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def _take(self, count: int, with_items: bool = False):
        buf = (Relation * max(count, 1))()
        its = (ctypes.c_uint32 * max(count, 1))() if with_items else None
        n = ctypes.c_size_t()
        self._check(self.lib.mps_take_relations(self.ctx, buf, its, count, ctypes.byref(n)))
        return buf, its, n.value

    def _relations(self, fn, *args, cap: int = 1 << 14):
        buf = (Relation * max(cap, 1))()
        n = ctypes.c_size_t()
        rc = fn(self.ctx, *args, buf, cap, ctypes.byref(n))
        if rc == MPS_E_CAPACITY:                      # fetch the kept result, no recomputation
            buf, _, _ = self._take(n.value)
        else:
            self._check(rc)
        return [(buf[i].p, buf[i].M, buf[i].q) for i in range(n.value)]

    def chunk_relations(self, lo: int, hi: int, item: Item):
        return self._relations(self.lib.mps_chunk_relations, lo, hi, ctypes.byref(item))

    def item_relations(self, item: Item):
        return self._relations(self.lib.mps_item_relations, ctypes.byref(item))

    def sieve_filter(self, lo: int, hi: int, item: Item, cap: int = 1 << 14) -> list[int]:
        while True:
            buf = (ctypes.c_uint64 * max(cap, 1))()
            n = ctypes.c_size_t()
            rc = self.lib.mps_sieve_filter(self.ctx, lo, hi, ctypes.byref(item), buf, cap, ctypes.byref(n))
            if rc == MPS_E_CAPACITY:
                cap = n.value
                continue
            self._check(rc)
            return list(buf[:n.value])

    def filter(self, primes: list[int], item: Item) -> list[int]:
        n = len(primes)
        arr = (ctypes.c_uint64 * max(n, 1))(*primes)
        flags = (ctypes.c_uint8 * max(n, 1))()
        self._check(self.lib.mps_filter(self.ctx, arr, n, ctypes.byref(item), flags))
        return list(flags[:n])

    def batch_relations(self, items: list[Item], cap: int = 1 << 14):
        arr = (Item * max(len(items), 1))(*items)
        buf = (Relation * max(cap, 1))()
        its = (ctypes.c_uint32 * max(cap, 1))()
        n = ctypes.c_size_t()
        rc = self.lib.mps_batch_relations(self.ctx, arr, len(items), buf, its, cap, ctypes.byref(n))
        if rc == MPS_E_CAPACITY:
            buf, its, _ = self._take(n.value, with_items=True)
        else:
            self._check(rc)
        return [(its[i], buf[i].p, buf[i].M, buf[i].q) for i in range(n.value)]

    def count_primes(self, lo: int, hi: int) -> int:
        c = ctypes.c_uint64()
        self._check(self.lib.mps_count_primes(self.ctx, lo, hi, ctypes.byref(c)))
        return c.value

    def measure_peaks(self) -> dict:
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mps_measure_peaks(self.ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        d = ctypes.c_double()
        self._check(self.lib.mps_measure_smem_peak(self.ctx, ctypes.byref(d)))
        return {"fp64_mulmod_per_s": a.value, "int_mulmod_per_s": b.value, "imad_per_s": c.value,
                "smem_atomic_per_s": d.value}

    def autotune(self, items: list[Item]) -> list[dict]:
        """Tunes the BSGS configuration of every item class among items (mps_autotune)."""
        arr = (Item * max(len(items), 1))(*items)
        n = ctypes.c_size_t()
        cap = max(len(items), 1)
        out = (TuneReport * cap)()
        self._check(self.lib.mps_autotune(self.ctx, arr, len(items), out, cap, ctypes.byref(n)))
        return [{k: getattr(out[i], k) for k, _ in TuneReport._fields_} for i in range(n.value)]

    def tune_save(self, path: str):
        self._check(self.lib.mps_tune_save(self.ctx, path.encode()))

    def tune_load(self, path: str):
        self._check(self.lib.mps_tune_load(self.ctx, path.encode()))

    def tune_clear(self):
        self._check(self.lib.mps_tune_clear(self.ctx))

    def survivors(self, lo: int, hi: int, cap: int = 1 << 16) -> list[int]:
        while True:
            buf = (ctypes.c_uint64 * max(cap, 1))()
            n = ctypes.c_size_t()
            rc = self.lib.mps_test_survivors(self.ctx, lo, hi, buf, cap, ctypes.byref(n))
            if rc == MPS_E_CAPACITY:
                cap = n.value
                continue
            self._check(rc)
            return list(buf[:n.value])

    def is_prime(self, nums: list[int]) -> list[int]:
        n = len(nums)
        arr = (ctypes.c_uint64 * max(n, 1))(*nums)
        out = (ctypes.c_uint8 * max(n, 1))()
        self._check(self.lib.mps_test_is_prime(self.ctx, arr, n, out))
        return list(out[:n])

    def bsgs(self, cases: list[tuple[int, int, int, int, int]], table_bits: int = 12) -> list[int | None]:
        flat = [x for c in cases for x in c]
        arr = (ctypes.c_uint64 * max(len(flat), 1))(*flat)
        out = (ctypes.c_uint64 * max(len(cases), 1))()
        self._check(self.lib.mps_test_bsgs(self.ctx, arr, len(cases), table_bits, out))
        return [None if out[i] == U64_MAX else out[i] for i in range(len(cases))]

    def order(self, pairs: list[tuple[int, int]]) -> list[int]:
        flat = [x for bp in pairs for x in bp]
        arr = (ctypes.c_uint64 * max(len(flat), 1))(*flat)
        out = (ctypes.c_uint64 * max(len(pairs), 1))()
        self._check(self.lib.mps_test_order(self.ctx, arr, len(pairs), out))
        return list(out[:len(pairs)])


class Server:
    """Continuous-batching server (mps_serve_*): submit items, wait for them."""

    def __init__(self, device: int = 0, tuning: Tuning | None = None, **cfg):
        self.lib = load_library()
        conf = ServeConfig()
        self.lib.mps_serve_config_default(ctypes.byref(conf))
        for k, v in cfg.items():
            setattr(conf, k, v)
        if tuning is None:
            tuning = default_tuning()
        self.sv = ctypes.c_void_p()
        rc = self.lib.mps_serve_open(device, ctypes.byref(tuning), ctypes.byref(conf), ctypes.byref(self.sv))
        if rc != MPS_OK:
            raise MpsError(rc, "mps_serve_open failed")

    def submit(self, item: Item) -> int:
        t = ctypes.c_uint64()
        rc = self.lib.mps_serve_submit(self.sv, ctypes.byref(item), ctypes.byref(t))
        if rc != MPS_OK:
            raise MpsError(rc, "submit")
        return t.value

    def wait(self, ticket: int, timeout: float = 600.0) -> dict:
        st = ServeStatus()
        rc = self.lib.mps_serve_wait(self.sv, ticket, timeout, ctypes.byref(st))
        if rc not in (MPS_OK, MPS_E_TIMEOUT):
            raise MpsError(rc, f"ticket {ticket} failed")
        return {k: getattr(st, k) for k, _ in ServeStatus._fields_} | {"done": rc == MPS_OK}

    def result(self, ticket: int):
        n = ctypes.c_size_t()
        rc = self.lib.mps_serve_result(self.sv, ticket, None, 0, ctypes.byref(n))
        if rc not in (MPS_OK, MPS_E_CAPACITY):
            raise MpsError(rc, f"result {ticket}")
        buf = (Relation * max(n.value, 1))()
        rc = self.lib.mps_serve_result(self.sv, ticket, buf, n.value, ctypes.byref(n))
        if rc != MPS_OK:
            raise MpsError(rc, f"result {ticket}")
        return [(buf[i].p, buf[i].M, buf[i].q) for i in range(n.value)]

    def release(self, ticket: int):
        self.lib.mps_serve_release(self.sv, ticket)

    def checkpoint(self, ticket: int) -> tuple[int, int]:
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        rc = self.lib.mps_serve_checkpoint(self.sv, ticket, ctypes.byref(a), ctypes.byref(b))
        if rc != MPS_OK:
            raise MpsError(rc, "checkpoint")
        return a.value, b.value

    def pool(self) -> dict:
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        c, d = ctypes.c_uint32(), ctypes.c_uint32()
        rc = self.lib.mps_serve_pool(self.sv, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d))
        if rc != MPS_OK:
            raise MpsError(rc, "pool")
        return {"pool_bytes": a.value, "reserved_bytes": b.value, "active": c.value, "queued": d.value}

    def close(self):
        if self.sv:
            self.lib.mps_serve_close(self.sv)
            self.sv = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
