"""The serving loop: items submitted while others run are admitted and batched
together; each result equals the item alone (and the reference's golden
relations)."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def _cases(golden, names_prefix=("c4_",), extra=("c2_low", "c3_low", "selftest", "small_p_2", "mod48", "b_128bit",
                                                   "empty_class")):
    return [c for c in golden["cases"] if c["name"].startswith(names_prefix) or c["name"] in extra]


def test_mix_equals_alone_and_golden(mps_lib, golden):
    cases = _cases(golden)
    items = [mps_lib.make_item(*c["item"]) for c in cases]
    with mps_lib.Server(0, max_active=8, piece_odds=1 << 18) as sv:
        # alone: one item at a time
        alone = []
        dense = [k for k, c in enumerate(cases) if c["relations"]][:6]
        for it in [items[k] for k in dense]:
            t = sv.submit(it)
            st = sv.wait(t)
            assert st["done"] and st["state"] == 2
            alone.append(sv.result(t))
            sv.release(t)
        # in the mix: all submitted at once (more than max_active: some wait in the queue)
        tickets = [sv.submit(it) for it in items]
        mixed = []
        for t in tickets:
            st = sv.wait(t)
            assert st["done"], st
            assert st["latency_ms"] >= st["queue_ms"] >= 0
            p_done, n_rel = sv.checkpoint(t)
            res = sv.result(t)
            assert n_rel == len(res)
            mixed.append(res)
    for k, c in enumerate(cases):
        assert [list(r) for r in mixed[k]] == c["relations"], c["name"]
    assert len(alone) == 6
    for a, k in zip(alone, dense):
        assert a == mixed[k] and a, cases[k]["name"]


def test_checkpoint_progress_on_device(mps_lib):
    """A long item's device-resident progress advances while it runs."""
    it = mps_lib.make_item(10, 111, 10**12, 10**12 + 2 * 10**9, 0, 10**7, 6, 4)
    with mps_lib.Server(0, piece_odds=1 << 22) as sv:
        t = sv.submit(it)
        seen = []
        while True:
            st = sv.wait(t, timeout=0.01)
            p_done, _ = sv.checkpoint(t)
            seen.append(p_done)
            if st["done"]:
                break
        assert seen[-1] == 10**12 + 2 * 10**9
        assert all(a <= b for a, b in zip(seen, seen[1:]))


def test_bad_item_is_rejected_at_submit(mps_lib):
    with mps_lib.Server(0) as sv:
        with pytest.raises(mps_lib.MpsError):
            sv.submit(mps_lib.make_item(2, -25, 100, 10, 0, 10, 1, 0))
        t = sv.submit(mps_lib.make_item(2, -25, 10**6, 10**6 + 10**5, 0, 1000, 1, 0))
        assert sv.wait(t)["done"]


def test_admission_waits_for_a_reservation(mps_lib, golden):
    """Admission is by the device pool: with room for two reservations the
    third item waits in the queue until one of the first two has finished
    and released its buffer; every result still equals the golden one."""
    case = next(c for c in golden["cases"] if c["name"] == "c2_low")          # 2,364 relations
    it = mps_lib.make_item(*case["item"])
    want = [tuple(r) for r in case["relations"]]
    with mps_lib.Server(0, max_active=8, piece_odds=1 << 20) as sv:
        t = sv.submit(it)
        st = sv.wait(t)
        assert st["done"] and st["relations_on_device"] == 1
        assert sv.result(t) == want
        grain = (st["reserved_bytes"] + 255) // 256 * 256
    budget = 2 * grain + 1024
    with mps_lib.Server(0, max_active=8, mem_budget_bytes=budget, piece_odds=1 << 20) as sv:
        assert sv.pool()["pool_bytes"] == budget // 256 * 256
        tickets = [sv.submit(it) for _ in range(3)]
        seen_queued, max_active = 0, 0
        while True:
            pool = sv.pool()
            max_active = max(max_active, pool["active"])
            seen_queued = max(seen_queued, pool["queued"])
            if sv.wait(tickets[2], timeout=0.002)["done"]:
                break
        sts = [sv.wait(t) for t in tickets]
        assert max_active <= 2
        assert sts[2]["queue_ms"] >= min(sts[0]["latency_ms"], sts[1]["latency_ms"]) - 5.0
        for t in tickets:
            assert sv.result(t) == want
        assert sv.pool()["reserved_bytes"] == 0


def test_item_larger_than_the_pool_fails(mps_lib, golden):
    case = next(c for c in golden["cases"] if c["name"] == "c2_low")
    # a 16 KB pool: c2_low's reservation (~160 KB) never fits, an item with no
    # in-class exponent (the 256-relation minimum, 8 KB) does
    with mps_lib.Server(0, mem_budget_bytes=16384) as sv:
        t = sv.submit(mps_lib.make_item(*case["item"]))
        with pytest.raises(mps_lib.MpsError) as e:
            sv.wait(t)
        assert e.value.code == mps_lib.MPS_E_CAPACITY
        small = next(c for c in golden["cases"] if c["name"] == "empty_class")
        t2 = sv.submit(mps_lib.make_item(*small["item"]))             # the server keeps working
        assert sv.wait(t2)["done"] and sv.result(t2) == []


def test_checkpoint_counts_while_waves_overflow(mps_lib):
    """b^0 - 1 = 0: every prime gives a relation (M = 0), far more than a
    wave's relation buffer holds, so every wave is redone on the host path.
    The device-resident count stays consistent with the progress while the
    item runs, and the result equals the item alone."""
    it = mps_lib.make_item((1 << 80) + 3, -1, 10**9, 10**9 + 2 * 10**7, 0, 50_000, 2, 0)
    tun = mps_lib.default_tuning(chunk_odds=1 << 21)
    with mps_lib.Siever(0, tuning=tun) as s:
        alone = s.item_relations(it)
        nprimes = s.count_primes(10**9, 10**9 + 2 * 10**7)
    # every prime of the range except prime factors of b has the relation (p, 0, ord_p(b))
    assert nprimes - 3 <= len(alone) <= nprimes and all(M == 0 for _, M, _ in alone)
    polls = []
    with mps_lib.Server(0, tuning=tun, piece_odds=1 << 19) as sv:
        t = sv.submit(it)
        while True:
            st = sv.wait(t, timeout=0.005)
            if st["done"]:
                break
            polls.append(sv.checkpoint(t))
        got = sv.result(t)
    assert got == alone
    ps = [p for p, _, _ in got]
    import bisect
    for p_done, n_rel in polls:
        assert bisect.bisect_left(ps, p_done) <= n_rel <= len(got), (p_done, n_rel)
