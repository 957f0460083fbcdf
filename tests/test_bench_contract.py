"""bench.py's command line and its reference arm, on the CPU.

The reference arm times the reference's own CPU BFS on the host cores and
prints the same JSON line as the GPU arm with "impl": "reference"; under
torchrun only rank 0 prints.  The GPU arm itself needs a device and is run on
the GPU box.
"""
import io
import json
import os
import subprocess
import sys
import types
from contextlib import redirect_stdout

import pytest

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_defaults_are_one_gpu_and_a_short_run():
    old = sys.argv
    try:
        sys.argv = ["bench.py"]
        a = bench.parse()
    finally:
        sys.argv = old
    assert a.gpus == 1 and a.impl == "ours" and a.config == "rmat22"
    assert a.warmup >= 3 and a.steps >= 1 and a.levels == 0


def test_reference_arm_prints_one_json_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--config", "rmat20",
                          "--sources", "4", "--steps", "1", "--warmup", "0"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "GTEPS" and d["higher_is_better"] is True
    assert d["metric"] == bench.METRIC and d["value"] > 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_prints_nothing_on_other_ranks():
    args = types.SimpleNamespace(config="rmat20", sources=4, steps=1, warmup=0, gpus=2)
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args, rank=1)
    assert buf.getvalue() == ""
