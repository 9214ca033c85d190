"""The reference arm of bench.py (the CPU oracle on the host cores) prints
one JSON line on the same metric, unit and workload as the product's arm,
so the two lines can be compared; checked on a small grid. Its value is one
complete solve measured whole, and its steps are consecutive iteration
ranges of that solve, so steps x ms_per_step is the measured time."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line_matches_the_contract():
    sys.path.insert(0, ROOT)
    import bench
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "10",
                          "--steps", "4", "--warmup", "1", "--cpu-sample-iters", "3"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.metric_name(10)
    assert line["unit"] == "s" and line["higher_is_better"] is False
    assert line["config"]["workload"] == bench.workload_name(10, line["config"]["nz_blocks"])
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["steps"] == 4 and len(line["step_s"]) == 4
    assert abs(line["ms_per_step"] * 4 - line["value"] * 1e3) < 1e-6 * line["value"] * 1e3
    # the iteration ranges add up to the measured solve (less its copy-out tail)
    assert 0.5 * line["value"] <= sum(line["step_s"]) <= line["value"]
    assert line["iterations"] > 4 and "status 0" in line["cpu_baseline"]["sample"]
    assert line["config"] == bench.shared_config(10, line["config"]["nz_blocks"], line["config"]["unknowns"])
