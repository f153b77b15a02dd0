"""bench.py's reference arm on the CPU: the JSON line it prints for the
small configuration carries the fields the measurement contract names."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    from oracle import build as ob
    if not os.path.exists(ob.ref_lib_path("sceptic")):
        try:
            ob.build_ref()
        except FileNotFoundError as e:
            pytest.skip(str(e))
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "small",
                        "--steps", "4", "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "particle-steps/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 4 and line["warmup"] == 3
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert "timed steps" in cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert line["config"]["N"] == 8193
