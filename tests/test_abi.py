"""The C-ABI library: builds for sm_100a, loads without a GPU, exports every
symbol include/mps_gpu.h declares, and its structs match the header."""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

from conftest import ROOT


def test_exports_every_header_symbol(mps_lib):
    lib = mps_lib.load_library()
    names = mps_lib.header_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layout_matches_header(mps_lib):
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "mps_gpu.h"
int main(void) {
    printf("%zu %zu %zu %zu %zu %zu\n", sizeof(mps_item), sizeof(mps_relation), sizeof(mps_tuning),
           sizeof(mps_stats), offsetof(mps_item, mod), offsetof(mps_tuning, plain));
    return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    want = [ctypes.sizeof(mps_lib.Item), ctypes.sizeof(mps_lib.Relation), ctypes.sizeof(mps_lib.Tuning),
            ctypes.sizeof(mps_lib.Stats), mps_lib.Item.mod.offset, mps_lib.Tuning.plain.offset]
    assert [int(x) for x in out] == want


def test_abi_version_and_defaults(mps_lib):
    lib = mps_lib.load_library()
    assert lib.mps_abi_version() == 1
    t = mps_lib.default_tuning()
    assert t.struct_size == ctypes.sizeof(mps_lib.Tuning)
    assert t.chunk_odds == 1 << 26 and t.bsgs_warps == 4 and t.table_kind == 3


def test_open_without_device_is_an_error_not_a_crash(mps_lib):
    import torch
    if torch.cuda.is_available():
        return
    lib = mps_lib.load_library()
    ctx = ctypes.c_void_p()
    t = mps_lib.default_tuning()
    assert lib.mps_open(0, ctypes.byref(t), ctypes.byref(ctx)) == mps_lib.MPS_E_NODEV
    assert not ctx.value
