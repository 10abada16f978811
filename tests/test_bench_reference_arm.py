"""The bench's reference arm (`bench.py --impl reference`) runs on the host
alone: one small scene through the reference's own CPU build must print the
contract's JSON line."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_its_line():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libccref_f32.so")):
        pytest.skip("the reference's CPU build is absent (make -C oracle ref)")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1", "--n", "20000"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1])
    assert line["impl"] == "reference" and line["metric"] == "bodies/s" and line["value"] > 0
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "reference"
    assert line["config"]["pairs"] > 0
