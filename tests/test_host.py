"""The drop-in program mps_siever: worktodo/prime.ini handling, relations ->
results.json (checked against a test-only Python restatement of
Worker.hpp:527-559 apply_relations and Results.hpp:72-140
append_results_json), and on the GPU a whole run in a scratch directory,
including resume from an interrupted run's checkpoint files."""
from __future__ import annotations

import json
import os
import random
import subprocess

import pytest

from conftest import PKG, ROOT

BIN = os.path.join(PKG, "mps_siever")
FAULTS_BIN = os.path.join(PKG, "mps_siever_faults")
INT64_MAX = 2**63 - 1
INT64_MIN = -(2**63)


def _build(target):
    srcs = [os.path.join(PKG, "host", f) for f in os.listdir(os.path.join(PKG, "host"))]
    srcs.append(os.path.join(ROOT, "include", "mps_gpu.h"))
    path = os.path.join(PKG, target)
    if not os.path.exists(path) or os.path.getmtime(path) < max(os.path.getmtime(f) for f in srcs):
        subprocess.run(["make", "-s", "-C", PKG, target], check=True)
    return path


@pytest.fixture(scope="session")
def siever_bin():
    return _build("mps_siever")


@pytest.fixture(scope="session")
def faults_bin():
    return _build("mps_siever_faults")


# ---------------------------------------------------- test-only restatement --

def _trunc_mod(a: int, m: int) -> int:
    """C++ `%` (truncating) on 128-bit integers."""
    r = abs(a) % m
    return -r if a < 0 else r


def _in_class(mod, res, n):                          # Types.hpp:28-31
    if mod <= 1:
        return True
    return (_trunc_mod(n, mod) % 2**64) == res


def _ceil_div(a, b):
    return -((-a) // b)


def _apply(item, relations):                         # Worker.hpp:527-559
    b, c, P0, P1, N0, N1, mod, res = item
    cand = [[] for _ in range(N1 - N0)]
    for p, M, q in relations:
        for x in range(_ceil_div(N0 - M, q), (N1 - 1 - M) // q + 1):
            n = q * x + M
            idx = n - N0
            if idx < 0 or idx >= len(cand):
                continue
            value, fits, e = 1, True, 0
            while e < n and fits:
                value *= b
                if value > 2 * p:
                    fits = False
                e += 1
            if fits and value + c == p:
                continue
            cand[idx].append(p)
    return cand


def _jint(v):
    return str(v) if v > INT64_MAX or v < INT64_MIN else v


def _entry(item, relations, ts):                     # Results.hpp:72-107
    b, c, P0, P1, N0, N1, mod, res = item
    cand = _apply(item, relations)
    prp, factored = [], []
    for i, f in enumerate(cand):
        n = N0 + i
        if not _in_class(mod, res, n):
            continue
        if not f:
            prp.append(_jint(n))
        else:
            factored.append({"n": _jint(n), "factors": [_jint(x) for x in f]})
    return {"Timestamp": ts, "b": _jint(b), "c": _jint(c), "P0": _jint(P0), "P1": _jint(P1), "N0": _jint(N0),
            "N1": _jint(N1), "prp": prp, "factored": factored}


def _dump(v):
    return json.dumps(v, separators=(",", ":"))


def _factor_line(item):
    b, c, P0, P1, N0, N1, mod, res = item
    return f"Factor={b},{c},{P0},{P1},{N0},{N1},{mod},{res}"


def _run_entry(bin_path, tmp_path, item, relations, ts="2026-12-03 01:02:03 UTC+0", results=None):
    rel = tmp_path / "rel.p"
    rel.write_text("".join(f"{p}, {M}, {q}\n" for p, M, q in relations))
    args = [bin_path, "--results-entry", str(rel), _factor_line(item), ts]
    if results is not None:
        args.append(str(results))
    out = subprocess.run(args, capture_output=True, text=True, check=True)
    return out.stdout.strip()


# ---------------------------------------------------------------- CPU tests --

def test_entry_random(siever_bin, tmp_path):
    rng = random.Random(7)
    for _ in range(60):
        b = rng.choice([2, 3, 5, 6, 7, 10, 12])
        c = rng.choice([-1, 1]) * rng.randint(1, 999)
        N0 = rng.randint(-50, 3000)
        N1 = N0 + rng.randint(1, 400)
        mod = rng.choice([1, 2, 3, 6, 12])
        item = (b, c, 10**6, 10**7, N0, N1, mod, rng.randrange(mod))
        rels = [(rng.randint(3, 10**9), rng.randint(max(0, N0 - 100), N1 + 100), rng.randint(1, 60))
                for _ in range(rng.randint(0, 25))]
        assert _run_entry(siever_bin, tmp_path, item, rels) == _dump(_entry(item, rels, "2026-12-03 01:02:03 UTC+0"))


def test_entry_value_is_the_prime(siever_bin, tmp_path):
    # b^n + c == p is not a factorisation (10^2 + 111 = 211, 2^5 - 25 = 7)
    for item, rels in [((10, 111, 100, 1000, 0, 30, 1, 0), [(211, 2, 5)]),
                       ((2, -25, 3, 100, 0, 40, 2, 1), [(7, 5, 3), (23, 1, 11)])]:
        got = json.loads(_run_entry(siever_bin, tmp_path, item, rels))
        want = _entry(item, rels, got["Timestamp"])
        assert got == want
        assert all(f["n"] != 2 for f in got["factored"]) if item[0] == 10 else True


def test_entry_wide_integers(siever_bin, tmp_path):
    # 128-bit b, c and N0 outside int64 are written as strings; so are factors above 2^63-1
    item = (2**70 + 1, -(2**65) - 3, 10**12, 10**12 + 10**6, 2**63 + 5, 2**63 + 25, 1, 0)
    rels = [(2**63 + 29, 2**63 + 8, 4), (18446744073709551557, 2**63 + 10, 7), (1000003, 2**63 + 12, 1)]
    got = _run_entry(siever_bin, tmp_path, item, rels)
    assert got == _dump(_entry(item, rels, "2026-12-03 01:02:03 UTC+0"))
    assert '"b":"1180591620717411303425"' in got


def test_results_json_appends(siever_bin, tmp_path):
    results = tmp_path / "results.json"
    results.write_text('[{"x":"a\\"b\\\\c\\u00e9\\ud83d\\ude00","y":[1,-2,3.5e2,true,false,null],"z":{}}]\n')
    item = (2, -25, 10**6, 10**8, 0, 50, 2, 1)
    rels = [(1000003, 3, 7), (1000033, 9, 10)]
    _run_entry(siever_bin, tmp_path, item, rels, results=results)
    _run_entry(siever_bin, tmp_path, item, rels, ts="2026-12-03 01:02:04 UTC+0", results=results)
    text = results.read_text()
    assert text.endswith("\n") and "\n" not in text[:-1]
    data = json.loads(text)
    assert len(data) == 3
    assert data[0] == {"x": "a\"b\\cé\U0001F600", "y": [1, -2, 350.0, True, False, None], "z": {}}
    assert data[1] == _entry(item, rels, "2026-12-03 01:02:03 UTC+0")
    assert data[2]["Timestamp"] == "2026-12-03 01:02:04 UTC+0"


def test_results_json_not_an_array(siever_bin, tmp_path):
    results = tmp_path / "results.json"
    results.write_text('{"a": 1}')
    rel = tmp_path / "rel.p"
    rel.write_text("")
    r = subprocess.run([siever_bin, "--results-entry", str(rel), "Factor=2,-25,10,100,0,10", "t", str(results)],
                       capture_output=True, text=True)
    assert r.returncode == 1
    assert "results.json must contain a JSON array" in r.stderr


@pytest.mark.parametrize("line,message", [
    ("Factor=2,-25,10,100,0", "must have 6 or 8 comma-separated values (b,c,P0,P1,N0,N1[,mod,res])"),
    ("Factor=2,-25,100,10,0,10", "requires P0 < P1"),
    ("Factor=2,-25,10,100,10,10", "requires N0 < N1"),
    ("Factor=2,-25,10,100,0,10000001", "range N1-N0 exceeds 10 million"),
    ("Factor=2,-25,10,100,0,10,2,2", "parse error"),
    ("Factor=2,-2x5,10,100,0,10", "parse error"),
    ("# only a comment", "No work items found in worktodo.txt"),
])
def test_worktodo_errors(siever_bin, tmp_path, line, message):
    (tmp_path / "worktodo.txt").write_text(line + "\n")
    r = subprocess.run([siever_bin], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert message in r.stderr
    assert "[FATAL]" in (tmp_path / "siever.log").read_text()


def test_prime_ini_written(siever_bin, tmp_path):
    # prime.ini missing: written with the four keys; then the worktodo is read (here: missing -> fatal)
    r = subprocess.run([siever_bin], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert "Failed to open worktodo file: worktodo.txt" in r.stderr
    keys = [l.split("=")[0] for l in (tmp_path / "prime.ini").read_text().splitlines()]
    assert keys == ["CPU_count", "MemoryAllowed", "UseGPU", "GPU_device"]
    # an existing complete prime.ini is left as it is
    ini = "CPU_count=4\nMemoryAllowed=512\nUseGPU=1\nGPU_device=0\nGPU_strict=1\n"
    (tmp_path / "prime.ini").write_text(ini)
    subprocess.run([siever_bin], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert (tmp_path / "prime.ini").read_text() == ini


def test_factor_numbers_in_hex_and_octal(siever_bin, tmp_path):
    # the reference reads b..N1 with its 128-bit type's string reading: "0x" hex, leading-0 octal
    got = json.loads(_run_entry_line(siever_bin, tmp_path, "Factor=0x2,-031,0100,0x3e8,00,012,2,1"))
    assert (got["b"], got["c"], got["P0"], got["P1"], got["N0"], got["N1"]) == (2, -25, 64, 1000, 0, 10)
    assert got["prp"] == [1, 3, 5, 7, 9]


def _run_entry_line(bin_path, tmp_path, line, relations=()):
    rel = tmp_path / "rel.p"
    rel.write_text("".join(f"{p}, {M}, {q}\n" for p, M, q in relations))
    out = subprocess.run([bin_path, "--results-entry", str(rel), line, "t"], capture_output=True, text=True,
                         check=True)
    return out.stdout.strip()


def test_gpu_strict_without_device(siever_bin, tmp_path):
    # no usable device (an index no machine has): GPU_strict stops with the reference's message
    (tmp_path / "prime.ini").write_text("CPU_count=1\nMemoryAllowed=64\nUseGPU=1\nGPU_device=999\nGPU_strict=1\n")
    (tmp_path / "worktodo.txt").write_text("Factor=2,-25,1000000,2000000,0,1000,2,1\n")
    r = subprocess.run([siever_bin], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "[FATAL] GPU_strict=1 but no usable GPU backend; not sieving on the CPU" in r.stderr
    assert not (tmp_path / "results.json").exists()


def test_bad_prime_ini_value(siever_bin, tmp_path):
    # std::stoi's error escapes to main, as in the reference (Siever.cpp:209-211)
    (tmp_path / "prime.ini").write_text("CPU_count=four\nMemoryAllowed=64\n")
    r = subprocess.run([siever_bin], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert "[FATAL] Unhandled exception: stoi" in r.stderr


def test_malformed_relation_line(siever_bin, tmp_path):
    rel = tmp_path / "rel.p"
    rel.write_text("1000003, 5, 7\nnot a relation\n")
    r = subprocess.run([siever_bin, "--results-entry", str(rel), "Factor=2,-25,10,100,0,10", "t"],
                       capture_output=True, text=True)
    assert r.returncode == 1
    assert "Malformed relation line: not a relation" in r.stderr


# ---------------------------------------------------------------- GPU tests --

def _golden_case(golden, predicate):
    for case in golden["cases"]:
        if predicate(case):
            return case
    raise LookupError


def _write_job(tmp_path, items, memory_mb=64, cpu=1):
    (tmp_path / "prime.ini").write_text(f"CPU_count={cpu}\nMemoryAllowed={memory_mb}\nUseGPU=1\nGPU_device=0\n")
    (tmp_path / "worktodo.txt").write_text("".join(_factor_line(it) + "\n" for it in items))


def _parse_relations(text):
    out = []
    for line in text.splitlines():
        if line.strip():
            p, M, q = (int(x) for x in line.split(","))
            out.append((p, M, q))
    return out


@pytest.mark.gpu
def test_run_two_items(siever_bin, tmp_path, oracle, golden):
    from oracle.oracle import make_item as oracle_item

    items = [(2, -25, 10**9, 10**9 + 2 * 10**8, 0, 100_000, 2, 1),
             (10, 111, 10**12, 10**12 + 5 * 10**7, 0, 10**7, 6, 4)]
    _write_job(tmp_path, items)
    r = subprocess.run([siever_bin], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    data = json.loads((tmp_path / "results.json").read_text())
    assert len(data) == 2
    for item, entry in zip(items, data):
        want_rel = oracle.relations(item[2], item[3], oracle_item(*item))
        assert entry == _entry(item, want_rel, entry["Timestamp"])
    # relations.p holds the last item's relations, in increasing p
    rel = _parse_relations((tmp_path / "relations.p").read_text())
    assert rel == oracle.relations(items[1][2], items[1][3], oracle_item(*items[1]))
    assert not [f for f in os.listdir(tmp_path) if f.startswith("core_")]
    assert "Final status:" in r.stderr


@pytest.mark.gpu
def test_resume_after_interruption(siever_bin, tmp_path, oracle):
    """A run stopped after some chunks (core file + progress record written,
    plus relations of a chunk whose progress was never recorded) resumes at
    the recorded p and ends with the same relations.p and results entry."""
    from oracle.oracle import make_item as oracle_item

    item = (2, -25, 10**9, 10**9 + 3 * 10**8, 0, 100_000, 2, 1)
    want = oracle.relations(item[2], item[3], oracle_item(*item))
    stop = 10**9 + 10**8
    torn = 10**9 + 12 * 10**7
    _write_job(tmp_path, [item], cpu=2)
    core = [r for r in want if r[0] < torn]            # a chunk past `stop` half written
    (tmp_path / "core_2.p").write_text("".join(f"{p}, {M}, {q}\n" for p, M, q in core))
    b, c, P0, P1, N0, N1, mod, res = item
    (tmp_path / "core_progress.txt").write_text(f"{b} {c} {P0} {P1} {N0} {N1} {mod} {res} {stop}\n")
    r = subprocess.run([siever_bin], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert f"Checkpoint recovered: new P0 = {stop}" in r.stderr
    assert _parse_relations((tmp_path / "relations.p").read_text()) == want
    entry = json.loads((tmp_path / "results.json").read_text())[0]
    assert entry == _entry(item, want, entry["Timestamp"])
    assert entry["P0"] == item[2]


@pytest.mark.gpu
def test_resume_reference_checkpoint(siever_bin, tmp_path, oracle):
    """Core files written by the reference's own workers (no progress
    record): resume at the smallest last p, as the reference does."""
    from oracle.oracle import make_item as oracle_item

    item = (2, -25, 10**9, 10**9 + 10**8, 0, 100_000, 2, 1)
    want = oracle.relations(item[2], item[3], oracle_item(*item))
    assert len(want) > 40
    _write_job(tmp_path, [item], cpu=2)
    (tmp_path / "core_0.p").write_text("".join(f"{p}, {M}, {q}\n" for p, M, q in want[:10]))
    (tmp_path / "core_1.p").write_text("".join(f"{p}, {M}, {q}\n" for p, M, q in want[10:30]))
    r = subprocess.run([siever_bin], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert f"Checkpoint recovered: new P0 = {want[9][0]}" in r.stderr
    assert sorted(_parse_relations((tmp_path / "relations.p").read_text())) == want


def _entries_without_time(path):
    data = json.loads(path.read_text())
    for e in data:
        e.pop("Timestamp")
    return data


def _reference_run(siever_bin, tmp_path, items, memory_mb):
    ref = tmp_path / "uninterrupted"
    ref.mkdir()
    _write_job(ref, items, memory_mb=memory_mb)
    r = subprocess.run([siever_bin], cwd=ref, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return (ref / "relations.p").read_text(), _entries_without_time(ref / "results.json")


# two items, 2^24-integer chunks (MemoryAllowed=16 MB, CPU_count=1): 6 + 3 chunks
STOP_ITEMS = [(2, -25, 10**9, 10**9 + 10**8, 0, 100_000, 2, 1),
              (10, 111, 10**9, 10**9 + 5 * 10**7, 0, 10**7, 6, 4)]


@pytest.mark.gpu
def test_gpu_strict_declined_chunk_then_resume(siever_bin, faults_bin, tmp_path):
    """GPU_strict=1 and a chunk the device declines (injected on the host):
    the run stops as the reference's does (the INFO line naming the chunk,
    then FATAL "Worker pool failed", exit 1) with the finished chunks kept;
    the next run resumes and ends with the uninterrupted run's files."""
    want_rel, want_results = _reference_run(siever_bin, tmp_path, STOP_ITEMS, 16)
    run = tmp_path / "strict"
    run.mkdir()
    _write_job(run, STOP_ITEMS, memory_mb=16)
    with open(run / "prime.ini", "a") as f:
        f.write("GPU_strict=1\n")
    env = dict(os.environ, MPS_SIEVER_DECLINE_CHUNK="3")
    r = subprocess.run([faults_bin], cwd=run, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 1
    lo = 10**9 + 3 * (1 << 24)
    assert (f"[INFO] GPU_strict=1: the GPU sieve declined the chunk starting at {lo}; "
            "stopping instead of sieving on the CPU") in r.stderr
    assert r.stderr.rstrip().endswith("[FATAL] Worker pool failed")
    assert (run / "core_progress.txt").read_text().split()[-1] == str(lo)
    assert not (run / "results.json").exists()
    r = subprocess.run([siever_bin], cwd=run, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert f"Checkpoint recovered: new P0 = {lo}" in r.stderr
    assert (run / "relations.p").read_text() == want_rel
    assert _entries_without_time(run / "results.json") == want_results


@pytest.mark.gpu
@pytest.mark.parametrize("after", [0, 4, 7])
def test_sigint_between_chunks_then_resume(siever_bin, faults_bin, tmp_path, after):
    """SIGINT delivered between chunks (raised by the program itself after
    chunk `after`, through its real handler): the run ends with the
    checkpoint kept; the next run resumes to the uninterrupted run's
    relations.p and results.json.  A stop inside the second item (chunk 7)
    is resumed as with the reference: the finished first line is removed
    from worktodo.txt before the restart (every run redoes all listed items)."""
    want_rel, want_results = _reference_run(siever_bin, tmp_path, STOP_ITEMS, 16)
    run = tmp_path / "stopped"
    run.mkdir()
    _write_job(run, STOP_ITEMS, memory_mb=16)
    env = dict(os.environ, MPS_SIEVER_SIGNAL_AFTER=str(after))
    r = subprocess.run([faults_bin], cwd=run, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Shutdown: checkpoint preserved in core_*.p files" in r.stderr
    first_done = after >= 6                               # item 1 is chunks 0-5
    assert (run / "results.json").exists() == first_done
    if first_done:
        (run / "worktodo.txt").write_text(_factor_line(STOP_ITEMS[1]) + "\n")
    r = subprocess.run([siever_bin], cwd=run, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Checkpoint recovered: new P0 = " in r.stderr
    assert (run / "relations.p").read_text() == want_rel
    assert _entries_without_time(run / "results.json") == want_results
