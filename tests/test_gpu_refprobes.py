"""The reference's own operator probes (ZKX/test_all/operators: the radartools probe and the
firfilter2 / hilbert / upfirdn / resample_poly probes), compiled unmodified against this
repository's include/ by `make -C oracle probes` and linked to libzkx_rd.so, run here as the
reference runs them.  Each probe calls the operator's *_device function (this library) and the
reference's *_typed_cpu function on the same deterministic inputs and writes both digests and
their distance; the CPU digest must equal the one the reference published for that command
line, and the GPU result must match it.

The probes are built only where the reference checkout is available; without them the tests
skip."""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROBES = os.path.join(ROOT, "oracle", "_ref", "probes")
PUBLISHED = json.load(open(os.path.join(ROOT, "tests", "golden", "published_digests.json"), encoding="utf-8"))
RADAR_OPS = ["pulse_compression", "pulse_doppler", "ca_cfar", "cfar_alpha", "ambgfun"]
FILTER_OPS = ["firfilter2", "hilbert", "upfirdn", "resample_poly"]
DTYPES = ["FP32", "FP16", "INT32", "INT16", "INT8"]


def probe_path(op: str) -> str:
    return os.path.join(PROBES, ("radartools_" + op) if op in RADAR_OPS else op)


def have_probes() -> bool:
    return all(os.path.exists(probe_path(op)) for op in RADAR_OPS + FILTER_OPS)


def cases():
    """(operator, argument dict, published CPU digest or None)."""
    out = []
    seen = set()
    for c in PUBLISHED:
        op, args = c["operator"], dict(c["args"])
        if op not in RADAR_OPS + FILTER_OPS:
            continue
        args["warmup"], args["measured"] = "1", "1"
        key = (op, json.dumps(args, sort_keys=True))
        if key in seen:
            continue
        seen.add(key)
        out.append((op, args, c["cpu_output_digest"]))
        if op in RADAR_OPS and args["dtype"] == "FP32":
            # the same shapes for the other element types the reference instantiates
            for dt in DTYPES[1:]:
                out.append((op, dict(args, dtype=dt), None))
    for dt in DTYPES:
        out.append(("ambgfun", {"dtype": dt, "n0": "64", "fs": "2", "prf": "1", "warmup": "1", "measured": "1"}, None))
    return out


CASES = cases()


def case_id(c):
    op, a, _ = c
    return op + "-" + "-".join(f"{k}{v}" for k, v in sorted(a.items()) if k not in ("warmup", "measured"))


def test_probes_bind_device_calls_to_this_library():
    """Every probe defines the cusignal *_device templates it calls from include/ (so they are
    this library's implementations) and imports the C entry points of libzkx_rd.so."""
    if not have_probes():
        pytest.skip("reference probes not built (needs the reference checkout)")
    if shutil.which("nm") is None:
        pytest.skip("nm not available")
    for op in RADAR_OPS + FILTER_OPS:
        exe = probe_path(op)
        defined = subprocess.run(["nm", "-C", "--defined-only", exe], capture_output=True, text=True).stdout
        undefined = subprocess.run(["nm", "-D", "--undefined-only", exe], capture_output=True, text=True).stdout
        device_fn = {"ca_cfar": "ca_cfar_device", "cfar_alpha": "cfar_alpha_device",
                     "ambgfun": "ambgfun_device"}.get(op, op + "_device")
        assert f"cusignal::{device_fn}<" in defined, (op, "device template not instantiated from include/")
        assert " zkx_" in undefined, (op, "no libzkx_rd.so entry point imported")


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[case_id(c) for c in CASES])
def test_reference_probe_passes_on_this_library(case):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not have_probes():
        pytest.skip("reference probes not built (needs the reference checkout)")
    op, args, published = case
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "raw.json")
        cmd = [probe_path(op)]
        for k, v in args.items():
            cmd += ["--" + k, str(v)]
        cmd += ["--output", out]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        raw = json.load(open(out))
    if published is not None:
        assert raw["cpu_output_digest"] == published, "the reference CPU function did not reproduce its digest"
    assert raw.get("semantic_check", True) in (True, "true", 1)
    if op == "ca_cfar":
        # thresholds and masks bit-identical to ca_cfar_typed_cpu
        assert raw["mismatch_count"] == 0
        assert raw["relative_l2"] == 0
        assert raw["gpu_output_digest"] == raw["cpu_output_digest"]
    else:
        assert raw["relative_l2"] <= 1e-5, raw["relative_l2"]
