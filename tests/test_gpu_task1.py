"""The reference's own Task1 radar pipeline (ZKX/Task1: LFM + echo synthesis, pulse
compression, pulse Doppler, |.|^2 + cfar_alpha + 2-D CA-CFAR, ambiguity function), every
source compiled UNCHANGED against this repository's include/ and linked to libzkx_rd.so
for each *_device call (`make -C oracle task1`), run on the reference's S11 configuration
([128, 512], the case whose console log the reference published,
ZKX/Task1/evidence/visualization/pipeline.log).

The pipeline checks itself as the reference wrote it: each step compares its GPU output
with the reference's own *_typed_cpu function (compiled from the reference, oracle/_ref)
and exits non-zero if any gate fails; step 4 requires the GPU detection mask to equal the
CPU CA-CFAR fed the same GPU power.  On top of that the semantic figures (detected range
and Doppler bins, CFAR alpha, missed targets, false alarms) are compared with the
published log; and the pipeline's formal benchmark, run on the ten S11 scales, writes the
reference's CSV evidence rows (task1_benchmark_*.csv: timing statistics, accuracy and
mismatch counts against an independent host pipeline), compared with the rows the reference
published for its own formal matrix.

The binaries are built only where the reference checkout is available; without them the
tests skip."""
from __future__ import annotations

import csv
import json
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
T1 = os.path.join(ROOT, "oracle", "_ref", "task1")
PIPELINE = os.path.join(T1, "task1_pipeline")
BENCHMARK = os.path.join(T1, "task1_pipeline_benchmark")
CONF = os.path.join(T1, "task1_selected.conf")
PUBLISHED = json.load(open(os.path.join(ROOT, "tests", "golden", "task1_s11_published.json"), encoding="utf-8"))
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


def parse_log(text: str) -> dict:
    steps: dict = {}
    summary: dict = {}
    for line in text.splitlines():
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
    return {"steps": steps, "summary": summary}


def _require_binaries(*paths):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    missing = [p for p in paths if not os.path.exists(p)]
    if missing:
        pytest.skip(f"Task1 binaries not built: {missing}")


def test_task1_pipeline_s11_matches_published_evidence(tmp_path):
    _require_binaries(PIPELINE, CONF)
    vis = tmp_path / "visualization"
    vis.mkdir()
    env = dict(os.environ, ZKX_VISUALIZATION_DIR=str(vis))
    r = subprocess.run([PIPELINE, "--config", CONF], cwd=tmp_path, env=env, capture_output=True,
                       text=True, timeout=600)
    print(r.stdout[-4000:])
    assert r.returncode == 0, r.stderr[-2000:]
    ours = parse_log(r.stdout)
    assert ours["summary"].get("status") == "pass"
    assert ours["summary"].get("accuracy_pass") == "5/5"
    for step in ("step1", "step2", "step3", "step4", "step5"):
        acc = ours["steps"][step]["accuracy"]
        pub = PUBLISHED["steps"][step]["accuracy"]
        assert acc["status"] == "pass", step
        assert acc["compared_elements"] == pub["compared_elements"], step
        assert acc["relative_l2_error"] <= pub["relative_tolerance"], step
    m = {s: ours["steps"][s]["metrics"] for s in ours["steps"]}
    p = {s: PUBLISHED["steps"][s]["metrics"] for s in PUBLISHED["steps"]}
    # semantic figures equal to the published run
    for step, key in [("step2", "peak_range_bin"), ("step2", "expected_range_bin"),
                      ("step2", "compressed_half_power_width_samples"),
                      ("step3", "peak_doppler_bin"), ("step3", "peak_range_bin"),
                      ("step3", "detected_doppler_hz"), ("step4", "target_detected"),
                      ("step4", "missed_targets"), ("step4", "target_doppler_index"),
                      ("step4", "pure_noise_false_alarms"), ("step4", "reference_cell_count"),
                      ("step5", "peak_delay_index"), ("step5", "peak_doppler_index"),
                      ("step5", "delay_mainlobe_width_samples")]:
        assert m[step][key] == p[step][key], (step, key, m[step][key], p[step][key])
    assert abs(m["step4"]["cfar_alpha"] - p["step4"]["cfar_alpha"]) <= 1e-6 * p["step4"]["cfar_alpha"]
    for key in ("delay_pslr_db", "doppler_pslr_db"):
        assert abs(m["step5"][key] - p["step5"][key]) <= 1e-3
    # false alarms come from the same scene; the count may move only by cells whose power
    # lies at the threshold to within the last bits of FP32
    assert abs(m["step4"]["false_alarms"] - p["step4"]["false_alarms"]) <= 3, m["step4"]["false_alarms"]
    # the reference-format evidence the runner writes
    ev = json.load(open(tmp_path / "task1_pipeline_evidence.json", encoding="utf-8"))
    assert ev["status"] == "pass" and ev["completed_steps"] == 5 and len(ev["steps"]) == 5
    assert (vis / "task1_manifest.csv").exists()


S11_SCALES = sorted(PUBLISHED["formal_s11"])


@pytest.mark.parametrize("scale_id", S11_SCALES)
def test_task1_pipeline_benchmark_matches_published_matrix(tmp_path, scale_id):
    """The reference's formal pipeline benchmark on one of the ten [128, 512] S11 scales
    (smoke run: 1 warm-up, 3 measured), against the row the reference published for it.
    Its CPU leg is the reference's own code on the same input, so when the scale's
    configuration digest equals the published one the input digest and the CPU output
    digest must be identical; the GPU leg must pass the benchmark's own gates (mask equal to
    the CPU CFAR fed the same GPU power), and its distance to the benchmark's independent
    host pipeline -- relative L2 and detection-mask mismatches, which that host pipeline's
    own FP32 error dominates -- must be the published GPU's (the published matrix used an
    earlier revision of the scale file: where the configuration digest differs, the scene's
    noise differs too and the mismatch counts agree only statistically)."""
    _require_binaries(BENCHMARK)
    out = tmp_path / "out"
    cmd = [BENCHMARK, "--task-scales", os.path.join(T1, "task_input_scales.json"),
           "--accuracy-thresholds", os.path.join(T1, "accuracy_thresholds.json"),
           "--scale-id", scale_id, "--backend", "unbound", "--run-id", "b200",
           "--run-type", "smoke", "--warmup-runs", "1", "--measured-runs", "3",
           "--output-dir", str(out)]
    r = subprocess.run(cmd, cwd=tmp_path, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    rows = list(csv.DictReader(open(out / "task1_benchmark_unbound_smoke.csv", encoding="utf-8")))
    ours = {row["device"]: row for row in rows}
    for row in csv.DictReader(open(out / "task1_iteration_timing_unbound_smoke.csv", encoding="utf-8")):
        ours[row["device"]].setdefault("input_digest", row["input_digest"])
        ours[row["device"]].setdefault("output_digest", row["output_digest"])
    pub = PUBLISHED["formal_s11"][scale_id]
    gpu, cpu = ours["gpu"], ours["cpu"]
    assert gpu["accuracy_status"] == "PASS" and gpu["exact_match"] == "true" and gpu["mismatch_count"] == "0"
    assert gpu["measured_runs"] == "3" and gpu["scale_id"] == scale_id
    n_ours = int(gpu["independent_pipeline_mismatch_count"])
    n_pub = int(pub["gpu"]["independent_pipeline_mismatch_count"])
    print(f"\n{scale_id}: GPU p50 {float(gpu['p50_ms']):.3f} ms (published {float(pub['gpu']['p50_ms']):.3f}), "
          f"CPU p50 {float(cpu['p50_ms']):.1f} ms (published {float(pub['cpu']['p50_ms']):.1f}); rel-L2 to the "
          f"independent host pipeline {float(gpu['relative_l2']):.3e} (published {float(pub['gpu']['relative_l2']):.3e}); "
          f"mask mismatches {n_ours} (published {n_pub}); config digest "
          f"{'equal' if gpu['config_sha256'] == pub['gpu']['config_sha256'] else 'differs'}")
    if gpu["config_sha256"] == pub["gpu"]["config_sha256"]:
        assert gpu["input_digest"] == pub["gpu"]["input_digest"]
        assert cpu["output_digest"] == pub["cpu"]["output_digest"]
    assert float(gpu["relative_l2"]) <= 1.5 * float(pub["gpu"]["relative_l2"]) + 1e-7
    if gpu["config_sha256"] == pub["gpu"]["config_sha256"]:
        assert abs(n_ours - n_pub) <= max(5, 0.05 * n_pub)
    else:
        # the published matrix ran an earlier revision of the scale file (other seeds for
        # some scales), so the scenes differ and the counts agree only statistically
        assert abs(n_ours - n_pub) <= max(5, 0.25 * n_pub)
    for name in ("task1_iteration_timing_unbound_smoke.csv", "task1_memory_trace_unbound_smoke.csv",
                 "task1_accuracy_details_unbound_smoke.csv"):
        assert (out / name).exists(), name
