"""Compile tests/cpp/dropin_probe.cu (the operator API) and tests/cpp/runtime_probe.cu (the
runtime headers) against include/ and libzkx_rd.so with nvcc."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def build(out_dir: str, name: str = "dropin_probe") -> str:
    exe = os.path.join(out_dir, name)
    lib_dir = os.path.join(ROOT, "zkx_dev_b200")
    cmd = ["nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include"), os.path.join(HERE, name + ".cu"),
           "-L", lib_dir, "-lzkx_rd", "-Xlinker", "-rpath=" + lib_dir, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe
