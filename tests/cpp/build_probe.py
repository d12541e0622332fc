"""Compile tests/cpp/dropin_probe.cu against include/ and libzkx_rd.so with nvcc."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def build(out_dir: str) -> str:
    exe = os.path.join(out_dir, "dropin_probe")
    lib_dir = os.path.join(ROOT, "zkx_dev_b200")
    cmd = ["nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "dropin_probe.cu"),
           "-L", lib_dir, "-lzkx_rd", "-Xlinker", "-rpath=" + lib_dir, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe
