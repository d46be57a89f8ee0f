"""The reference arm of bench.py on the host cores (no GPU needed): one JSON
line with the metric, unit and workload of the default arm, `impl` =
"reference", a `cpu_baseline` describing the run, and an `e2e` object with
no host<->device bytes (the reference path runs on the host)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_shear256x128x64")):
        pytest.skip("host-compiled reference binary not built")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "Mcell-updates/s" and d["unit"] == "Mcell-updates/s"
    assert d["higher_is_better"] is True and d["value"] > 0
    assert d["config"]["workload"] == "mri_shearing_box_128x256x64"
    assert d["steps"] == 1 and d["warmup"] >= 3 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
