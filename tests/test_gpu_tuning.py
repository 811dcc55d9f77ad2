"""The autotuner (mps_autotune): every candidate configuration gives the same
relations (checked inside the tuner), the chosen one reproduces the
reference-built golden relations, and the tuning cache round-trips."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu

NAMES = ("selftest", "c2_low", "c3_low", "b7_nomod", "b12_mod12", "mod48", "wide_n", "small_p_10", "b_128bit")


def test_tuned_relations_equal_golden(mps_lib, golden, tmp_path):
    cases = [c for c in golden["cases"] if c["name"] in NAMES]
    items = [mps_lib.make_item(*c["item"]) for c in cases]
    with mps_lib.Siever(0) as s:
        reports = s.autotune(items)
        assert reports and all(r["candidates"] >= 10 for r in reports)
        for r in reports:
            assert r["table_kind"] in (0, 2, 3) and r["chains"] in (1, 2, 4) and r["warps"] in (4, 8)
            assert 1 <= r["table_fill"] <= 256 and 1 <= r["baby_scale"] <= 1024
            assert r["best_ns_per_prime"] <= r["default_ns_per_prime"] * 1.0001
            assert r["seg_words"] in (1024, 2048, 4096) and r["lanes"] in (8, 16, 32)
        for c, it in zip(cases, items):
            assert [list(x) for x in s.item_relations(it)] == c["relations"], c["name"]
        got = s.batch_relations(items)
        for k, c in enumerate(cases):
            assert [[p, M, q] for i, p, M, q in got if i == k] == c["relations"], c["name"]
        path = str(tmp_path / "tune.txt")
        s.tune_save(path)
    text = open(path).read().splitlines()
    assert text[0] == "mps-tune 4" and len(text) == 1 + len(reports)
    with mps_lib.Siever(0) as s2:
        s2.tune_load(path)
        for c, it in zip(cases, items):
            assert [list(x) for x in s2.item_relations(it)] == c["relations"], c["name"]
        s2.tune_clear()


def test_tuning_file_with_bad_lines(mps_lib, tmp_path, golden):
    path = tmp_path / "tune.txt"
    # a kind, chain count, warp count, segment, lane split, fill or scale the kernels are not built for is skipped
    path.write_text("mps-tune 4\n1 9 2 2 4 2048 32 192 256 1.0\n2 2 2 3 4 2048 32 192 256 1.0\n"
                    "3 2 2 2 99 2048 32 192 256 1.0\n4 2 2 2 4 3000 32 192 256 1.0\n5 0 2 2 4 2048 8 192 256 1.0\n"
                    "6 2 2 4 4 2048 16 192 256 1.0\n7 0 2 2 4 2048 32 0 256 1.0\n8 3 2 2 4 2048 32 192 2000 1.0\n")
    case = next(c for c in golden["cases"] if c["name"] == "selftest")
    with mps_lib.Siever(0) as s:
        s.tune_load(str(path))
        assert [list(x) for x in s.item_relations(mps_lib.make_item(*case["item"]))] == case["relations"]
    (tmp_path / "bad.txt").write_text("not a tuning file\n")
    with mps_lib.Siever(0) as s:
        with pytest.raises(mps_lib.MpsError):
            s.tune_load(str(tmp_path / "bad.txt"))
