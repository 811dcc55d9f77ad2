"""P-range sharding across ranks (multi_gpu.py) on CPU: two gloo ranks, each
computing its slice with the oracle in place of its GPU, gather the
relations to rank 0; the merged relations.p and results.json equal the
single-run ones, and merge_results (kaggle/merge_results.py) of per-slice
results equals the whole-range entry's prp list."""
from __future__ import annotations

import json
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT, PKG

import multi_gpu
from test_host import _entry, siever_bin  # noqa: F401  (fixture)

SPEC = (2, -25, 10**6, 10**7, 0, 20_000, 2, 1)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_slice(lo, hi, spec):
    from oracle.oracle import Oracle, make_item
    b, c, _, _, N0, N1, mod, res = spec
    return Oracle().relations(lo, hi, make_item(b, c, lo, hi, N0, N1, mod, res), threads=2)


def _rank_main(rank: int, world: int, port: int, out_dir: str, bin_path: str, spec=SPEC):
    import datetime
    import sys
    for p in (ROOT, PKG):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist
    from oracle.oracle import Oracle, make_item

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        rels = multi_gpu.slice_relations(_oracle_slice, spec, world, rank)
        merged = multi_gpu.gather_relations(dist, rels, rank, world)
        if rank == 0:
            multi_gpu.write_outputs(out_dir, spec, merged, siever_bin=bin_path)
        else:
            assert merged is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_shard_bounds():
    assert multi_gpu.shard_bounds(10, 21, 3, 0) == (10, 13)
    assert multi_gpu.shard_bounds(10, 21, 3, 1) == (13, 16)
    assert multi_gpu.shard_bounds(10, 21, 3, 2) == (16, 21)
    for world in (1, 2, 3, 8):
        cuts = [multi_gpu.shard_bounds(5, 10**9 + 7, world, r) for r in range(world)]
        assert cuts[0][0] == 5 and cuts[-1][1] == 10**9 + 7
        assert all(a[1] == b[0] for a, b in zip(cuts, cuts[1:]))
    with pytest.raises(ValueError):
        multi_gpu.shard_bounds(0, 10, 2, 2)


def test_parse_factor_line():
    assert multi_gpu.parse_factor_line("Factor=2,-25,10,100,0,10") == (2, -25, 10, 100, 0, 10, 1, 0)
    assert multi_gpu.parse_factor_line(" 10, 111, 5, 9, 1, 3, 6, 4 ") == (10, 111, 5, 9, 1, 3, 6, 4)
    for bad in ("Factor=2,-25,10,100,0", "Factor=2,-25,100,10,0,10", "Factor=2,-25,10,100,0,10,2,2"):
        with pytest.raises(ValueError):
            multi_gpu.parse_factor_line(bad)


def test_merge_relations_rejects_overlap():
    with pytest.raises(ValueError):
        multi_gpu.merge_relations([[(7, 1, 3)], [(7, 1, 3)]])
    assert multi_gpu.merge_relations([[(11, 0, 1)], [(3, 1, 2), (5, 2, 4)]]) == [(3, 1, 2), (5, 2, 4), (11, 0, 1)]


def test_two_rank_gloo(siever_bin, tmp_path, oracle):  # noqa: F811
    from oracle.oracle import make_item
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path), siever_bin)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    want = oracle.relations(SPEC[2], SPEC[3], make_item(*SPEC))
    got = []
    for line in (tmp_path / "relations.p").read_text().splitlines():
        p, M, q = (int(x) for x in line.split(","))
        got.append((p, M, q))
    assert got == want
    entry = json.loads((tmp_path / "results.json").read_text())[0]
    assert entry == _entry(SPEC, want, entry["Timestamp"])


def test_two_rank_gloo_range_narrower_than_world(siever_bin, tmp_path, oracle):  # noqa: F811
    """A P range of one integer over two ranks: rank 0's slice is empty, it
    computes nothing and still joins the gather; the result is the whole item's."""
    from oracle.oracle import make_item
    spec = (2, -25, 1_000_037, 1_000_038, 0, 20_000, 1, 0)      # one prime
    world, port = 2, _free_port()
    assert multi_gpu.shard_bounds(spec[2], spec[3], world, 0) == (spec[2], spec[2])
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path), siever_bin, spec))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    want = oracle.relations(spec[2], spec[3], make_item(*spec))
    entry = json.loads((tmp_path / "results.json").read_text())[0]
    assert entry == _entry(spec, want, entry["Timestamp"])


def test_merge_results_of_slices(oracle):
    from oracle.oracle import make_item
    b, c, P0, P1, N0, N1, mod, res = SPEC
    files = []
    for r in range(3):
        lo, hi = multi_gpu.shard_bounds(P0, P1, 3, r)
        spec = (b, c, lo, hi, N0, N1, mod, res)
        files.append([_entry(spec, oracle.relations(lo, hi, make_item(*spec)), "t")])
    whole = _entry(SPEC, oracle.relations(P0, P1, make_item(*SPEC)), "t")
    merged = multi_gpu.merge_results(files)
    assert merged["survivors"] == whole["prp"]
    assert merged["gaps"] == []
    files[1][0]["P0"] += 1000                           # a slice that started late leaves a gap
    assert multi_gpu.merge_results(files)["gaps"] == [(files[0][0]["P1"], files[1][0]["P0"])]
    files[2][0]["N1"] += 1
    with pytest.raises(ValueError):
        multi_gpu.merge_results(files)
