"""Per-launch DRAM traffic of the stencil kernels from ncu CSV output, as the JSON that
``bench.py`` reports under ``roofline.traffic``.

    ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum \\
        --clock-control none --print-units base -k regex:efm_ -c N --csv --log-file t.csv CMD
    python -m elastic_fm_vp_vs_rho_b200.ncu_traffic --workload NAME t.csv > profiles/ncu_traffic.json

The JSON records the SHA-256 of the stencil kernels' sources (``STENCIL_SOURCES``) it was
captured with; ``bench.py`` reports the traffic only while they still hash the same, so a
stale capture shows up as ``traffic: null`` with a note instead of a silent old number.
"""
from __future__ import annotations

import argparse
import csv
import hashlib
import json
import os
import re
import statistics
import sys

CSRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc")

# ncu kernel names (demangled templates) -> the bench's kernel kinds
_KINDS = [
    (re.compile(r"efm_pair_stream<\s*1\s*,\s*2\b"), "adj_stress+rev_velocity"),
    (re.compile(r"efm_pair_stream<\s*2\s*,\s*1\b"), "rev_stress+adj_velocity"),
    (re.compile(r"efm_image_stream"), "imaging"),
    (re.compile(r"efm_stress_stream<\s*0\b"), "fwd_stress"),
    (re.compile(r"efm_velocity_stream<\s*0\b"), "fwd_velocity"),
    (re.compile(r"efm_stress_stream<\s*1\b"), "adj_stress"),
    (re.compile(r"efm_velocity_stream<\s*1\b"), "adj_velocity"),
    (re.compile(r"efm_stress_stream<\s*2\b"), "rev_stress"),
    (re.compile(r"efm_velocity_stream<\s*2\b"), "rev_velocity"),
]
_UNITS = {"byte": 1.0, "kbyte": 1e3, "mbyte": 1e6, "gbyte": 1e9, "tbyte": 1e12}


# the files that determine what the plane-streaming and imaging kernels read and write
STENCIL_SOURCES = ("efm_image.cu", "efm_internal.cuh", "efm_stream.cu", "efm_stream.cuh",
                   "efm_tma.cuh")


def sources_sha256() -> str:
    """SHA-256 over the stencil kernels' sources, in file-name order."""
    h = hashlib.sha256()
    for name in STENCIL_SOURCES:
        h.update(name.encode())
        with open(os.path.join(CSRC, name), "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def kind_of(kernel_name: str):
    for rx, kind in _KINDS:
        if rx.search(kernel_name):
            return kind
    return None


def parse(paths):
    """{kind: [bytes of each captured launch]} from ncu CSV files."""
    launches = {}
    for path in paths:
        with open(path, newline="") as f:
            lines = [ln for ln in f if ln.startswith('"')]  # skip ncu's own log lines
        for row in csv.DictReader(lines):
            kind = kind_of(row.get("Kernel Name", ""))
            name = row.get("Metric Name", "")
            if kind is None or name not in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
                continue
            unit = _UNITS.get(row.get("Metric Unit", "byte").strip().lower(), 1.0)
            val = float(row["Metric Value"].replace(",", "")) * unit
            launches.setdefault(kind, {}).setdefault(row["ID"], 0.0)
            launches[kind][row["ID"]] += val
    return {k: list(v.values()) for k, v in launches.items()}


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--workload", required=True)
    p.add_argument("--note", default="")
    p.add_argument("csv", nargs="+")
    a = p.parse_args(argv)
    per = parse(a.csv)
    out = {"workload": a.workload,
           "note": a.note or "dram__bytes_read.sum + dram__bytes_write.sum per launch (median of "
                             "the captured launches of each kind)",
           "sources_sha256": sources_sha256(),
           "launches_captured": {k: len(v) for k, v in per.items()},
           "bytes_per_launch": {k: int(statistics.median(v)) for k, v in per.items()}}
    json.dump(out, sys.stdout, indent=2)
    print()


if __name__ == "__main__":
    main()
