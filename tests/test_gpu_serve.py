"""The serving loop: items submitted while others run are admitted and batched
together; each result equals the item alone (and the reference's golden
relations)."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def _cases(golden, names_prefix=("c4_",), extra=("selftest", "small_p_2", "mod48", "b_128bit", "empty_class")):
    return [c for c in golden["cases"] if c["name"].startswith(names_prefix) or c["name"] in extra]


def test_mix_equals_alone_and_golden(mps_lib, golden):
    cases = _cases(golden)
    items = [mps_lib.make_item(*c["item"]) for c in cases]
    with mps_lib.Server(0, max_active=8, piece_odds=1 << 18) as sv:
        # alone: one item at a time
        alone = []
        for it in items[:6]:
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
        if k < len(alone):
            assert alone[k] == mixed[k], c["name"]


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
