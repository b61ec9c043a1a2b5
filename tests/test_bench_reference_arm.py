"""`bench.py --impl reference` on the CPU: the reference arm times the FP64 C
oracle (the port of the reference's CPU path) on the host cores and prints
one JSON line in the benchmark's format.  No GPU is involved, so the line's
contract is checked here: the metric and unit of the homs arm, what was
timed (spins, stride, median step time), the cpu_baseline record and an e2e
record with no host-device bytes."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.timeout(600)
def test_reference_arm_prints_its_line():
    res = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    line = json.loads(res.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == line["unit"] == "spin*sample*coil/s"
    assert line["higher_is_better"] is True and line["steps"] == 1 and line["warmup"] >= 3
    assert line["value"] > 0 and line["ms_per_step"] > 0
    cfg = line["config"]
    assert cfg["workload"].startswith("3d_stack_of_spirals_100x100x35_350000spins_32coils_4x9500adc")
    assert cfg["spins"] == cfg["spins_timed"] > 0 and cfg["stride"] >= 1 and cfg["extrapolated"] is False
    # the rate is what one step of the timed subsample gives
    units = cfg["spins"] * cfg["samples"] * cfg["coils"]
    assert line["value"] == pytest.approx(units / (line["ms_per_step"] / 1e3), rel=1e-9)
    base = line["cpu_baseline"]
    assert base["kind"] == "port" and base["cores"] >= 1 and base["value"] == line["value"]
    assert base["projection"]["extrapolated"] is True and base["projection"]["spins"] == 350000
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
