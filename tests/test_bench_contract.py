"""CPU test of bench.py's reference arm: one bounded evaluation of the
reference's own C path (oracle/_ref) on the host, and the JSON line the
driver reads from it: the arm's metric, unit and direction, a cpu_baseline
describing the run, and an e2e object with no host-device traffic."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ORACLE, ROOT


def test_reference_arm_json_line():
    if not os.path.exists(os.path.join(ORACLE, "_ref", "libephref.so")):
        pytest.skip("reference not built (make -C oracle)")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "force+logdet evals/s, 32x32 lattice Nt=64: mixed vs FP64 plain, same B200"
    assert line["unit"] == "evals/s" and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["value"] > 0
    assert abs(line["ms_per_step"] * line["value"] - 1e3) < 1e-6 * 1e3
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"] and cb["cores"] >= 1
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert line["config"]["workload"].startswith("32x32 triangular lattice")
