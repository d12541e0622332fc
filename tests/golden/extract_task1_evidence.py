"""Extract the reference's published Task1 pipeline evidence for its S11 configuration.

The reference ran its own Task1 pipeline (ZKX/Task1/pipeline/apps/pipeline/main.cu) on the
configuration ZKX/Task1/evidence/visualization/task1_selected.conf ([128, 512] pulses x
samples, "task1_s11_strong") and kept the console log beside it (pipeline.log).  Each
step prints one [TASK1][stepN][ACCURACY] line (its comparison against the reference's own
CPU functions, with a status) and [TASK1][METRIC] lines (semantic figures such as the
detected range bin, the CFAR alpha and the false-alarm count).

The reference also published its formal Task1 pipeline benchmark matrix
(plot_in_report/0817结果/0817结果（含耗时）/03_任务结果/Task1/formal/pipeline/fft_thrust: one
folder per scale with the rows of performance/cpp/pipeline_benchmark_main.cu).  For the ten
[128, 512] S11 scales the script keeps, per device, the input and output digests, the
timing statistics, the relative L2 against the benchmark's independent host pipeline and
its detection-mask mismatch counts.

This script reads both in place (it needs the reference checkout) and writes
``task1_s11_published.json`` beside itself; tests/test_gpu_task1.py compares the same
pipeline and benchmark, compiled against this repository's headers and library, with it.

    python tests/golden/extract_task1_evidence.py [--ref <ZKX_dev checkout>]

The checkout defaults to $ZKX_REFERENCE_ROOT, else a checkout named "reference" beside
this repository.
"""
from __future__ import annotations

import argparse
import csv
import glob
import json
import os
import re

LOG = os.path.join("ZKX", "Task1", "evidence", "visualization", "pipeline.log")
CONF = os.path.join("ZKX", "Task1", "evidence", "visualization", "task1_selected.conf")
FORMAL = os.path.join("plot_in_report", "0817结果", "0817结果（含耗时）", "03_任务结果", "Task1", "formal",
                      "pipeline", "fft_thrust")
KEEP = ["config_id", "config_sha256", "input_shape", "warmup_runs", "measured_runs", "mean_ms", "p50_ms",
        "p99_ms", "cpu_gpu_speedup", "relative_l2", "relative_linf", "exact_match", "mismatch_count",
        "independent_pipeline_mismatch_count", "independent_pipeline_valid_mismatch_count",
        "independent_pipeline_boundary_mismatch_count", "accuracy_status"]
FIELD = re.compile(r'(\w+)=("[^"]*"|\S+)')


def parse_fields(text: str) -> dict:
    out = {}
    for key, value in FIELD.findall(text):
        value = value.strip('"')
        try:
            out[key] = float(value)
        except ValueError:
            out[key] = value
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    here = os.path.dirname(os.path.abspath(__file__))
    ap.add_argument("--ref", default=os.environ.get("ZKX_REFERENCE_ROOT")
                    or os.path.normpath(os.path.join(here, "..", "..", "..", "reference")))
    opts = ap.parse_args()
    steps: dict = {}
    summary = {}
    with open(os.path.join(opts.ref, LOG), encoding="utf-8") as fh:
        for line in fh:
            m = re.match(r"\[TASK1\]\[(step\d)\]\[ACCURACY\] (.*)", line)
            if m:
                steps.setdefault(m.group(1), {})["accuracy"] = parse_fields(m.group(2))
                continue
            m = re.match(r"\[TASK1\]\[METRIC\] step=(step\d) name=(\S+) value=(\S+)", line)
            if m:
                steps.setdefault(m.group(1), {}).setdefault("metrics", {})[m.group(2)] = float(m.group(3))
                continue
            m = re.match(r"\[TASK1\]\[SUMMARY\] (.*)", line)
            if m:
                summary = parse_fields(m.group(1))
    config = {}
    with open(os.path.join(opts.ref, CONF), encoding="utf-8") as fh:
        for line in fh:
            line = line.strip()
            if line and not line.startswith("#") and "=" in line:
                k, v = line.split("=", 1)
                config[k] = float(v)
    formal = {}
    for case in sorted(glob.glob(os.path.join(opts.ref, FORMAL, "RB_*", "raw", "cases", "task1_s11_*"))):
        scale = os.path.basename(case)
        rows = {}
        with open(os.path.join(case, "task1_benchmark_fft_thrust_formal.csv"), encoding="utf-8") as fh:
            for r in csv.DictReader(fh):
                rows[r["device"]] = {k: r[k] for k in KEEP}
        with open(os.path.join(case, "task1_iteration_timing_fft_thrust_formal.csv"), encoding="utf-8") as fh:
            for r in csv.DictReader(fh):
                rows[r["device"]].setdefault("input_digest", r["input_digest"])
                rows[r["device"]].setdefault("output_digest", r["output_digest"])
        formal[scale] = rows
    out = {"source": LOG.replace(os.sep, "/"), "config": config, "steps": steps, "summary": summary,
           "formal_source": FORMAL.replace(os.sep, "/"), "formal_s11": formal}
    with open(os.path.join(here, "task1_s11_published.json"), "w", encoding="utf-8") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
        fh.write("\n")


if __name__ == "__main__":
    main()
