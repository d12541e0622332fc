"""The ctypes mirrors of the C ABI's structs (zkx_dev_b200/_lib.py) have the sizes and
field offsets that a C compiler gives the declarations in include/zkx_rd.h (no GPU)."""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess
import tempfile

import pytest

from zkx_dev_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "zkx_rd_desc": L.RdDesc,
    "zkx_resample_layout": L.ResampleLayout,
    "zkx_rd_server_desc": L.ServerDesc,
    "zkx_rd_request": L.Request,
    "zkx_rd_server_stats": L.ServerStats,
    "zkx_synth_target": L.SynthTarget,
    "zkx_rd_tuning": L.RdTuning,
    "zkx_rd_work_item": L.WorkItem,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_struct_layouts_match_header():
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "zkx_rd.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["return 0; }"]
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        with open(src, "w") as f:
            f.write("\n".join(lines))
        subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            cname, field, value = line.split()
            got[(cname, field)] = int(value)
    for cname, py in STRUCTS.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)
