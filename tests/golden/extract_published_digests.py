"""Extract the reference's published CPU-output digests for the radar-chain operators.

The reference's evidence archive (plot_in_report/0817结果/0817结果（含耗时）/04_算子结果) keeps,
for every operator probe run, the probe command line (``*_full.log``) and a raw JSON
with ``typed_input_manifest`` (SHA-256 of each input array) and ``cpu_output_digest``
(SHA-256 of the flattened output of the reference's ``*_typed_cpu`` function).  The
probe inputs are deterministic functions of the command-line arguments, so the oracle
can regenerate them and must reproduce both digests bit for bit.  firfilter2 and
hilbert (the remaining-operators probes) keep every element type.

This script reads the archive in place (it needs the reference checkout) and writes
``published_digests.json`` beside itself; tests/test_oracle_published.py consumes that
file without the reference.  Only FP32 cases are kept (the chain's arithmetic type).

    python tests/golden/extract_published_digests.py [--ref <ZKX_dev checkout>]

The checkout defaults to $ZKX_REFERENCE_ROOT, else a checkout named "reference" beside
this repository.
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import shlex

OPS = ["pulse_compression", "pulse_doppler", "ca_cfar", "cfar_alpha", "upfirdn",
       "resample_poly", "firfilter", "firfilter2", "hilbert"]
# operators whose cases are kept for every element type (their padding / output storage
# depends on it); the others keep FP32 only
ALL_DTYPES = {"firfilter2", "hilbert"}
ARCHIVE = os.path.join("plot_in_report", "0817结果", "0817结果（含耗时）", "04_算子结果")


def parse_command(log_path: str) -> dict:
    with open(log_path, encoding="utf-8") as fh:
        first = fh.readline().strip()
    if not first.startswith("command="):
        raise ValueError(f"no command line in {log_path}")
    argv = shlex.split(first[len("command="):])
    args = {}
    for i in range(1, len(argv) - 1, 2):
        if argv[i].startswith("--"):
            args[argv[i][2:]] = argv[i + 1]
    args.pop("output", None)
    return args


def main() -> None:
    ap = argparse.ArgumentParser()
    here = os.path.dirname(os.path.abspath(__file__))
    ap.add_argument("--ref", default=os.environ.get("ZKX_REFERENCE_ROOT")
                    or os.path.normpath(os.path.join(here, "..", "..", "..", "reference")))
    opts = ap.parse_args()
    root = os.path.join(opts.ref, ARCHIVE)
    cases = {}
    for op in OPS:
        for raw in sorted(glob.glob(os.path.join(root, "**", f"{op}_probe_raw.json"),
                                    recursive=True)):
            with open(raw, encoding="utf-8") as fh:
                d = json.load(fh)
            if d.get("requested_dtype") != "FP32" and op not in ALL_DTYPES:
                continue
            logs = glob.glob(os.path.join(os.path.dirname(raw), "*_full.log"))
            if not logs:
                continue
            args = parse_command(logs[0])
            key = op + "|" + json.dumps(args, sort_keys=True)
            entry = {
                "operator": op,
                "args": args,
                "typed_input_manifest": d["typed_input_manifest"],
                "cpu_output_digest": d["cpu_output_digest"],
                "source": os.path.relpath(raw, opts.ref),
            }
            prev = cases.get(key)
            if prev is not None and prev["cpu_output_digest"] != entry["cpu_output_digest"]:
                raise RuntimeError(f"conflicting published digests for {key}")
            cases.setdefault(key, entry)
    out = sorted(cases.values(), key=lambda e: (e["operator"], json.dumps(e["args"], sort_keys=True)))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "published_digests.json")
    with open(path, "w", encoding="utf-8") as fh:
        json.dump(out, fh, indent=1, ensure_ascii=False)
        fh.write("\n")
    print(f"wrote {len(out)} cases to {path}")


if __name__ == "__main__":
    main()
