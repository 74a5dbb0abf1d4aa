"""bench.py's reference arm on the CPU: `--impl reference` times the CPU restatement of the
reference on pairs of the device arm's batch and prints one JSON line with the same metric, unit
and config as the device arm (both come from bench_config), a cpu_baseline block and an e2e block
without transfers."""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_reference_arm_line_matches_the_device_arm_config():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "rgbd-flow_b200"))
    import bench
    import rgbdflow as rf
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "pairs/s" and line["higher_is_better"] is True
    assert line["config"] == bench.bench_config(rf, 16, 1)
    assert line["value"] > 0 and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
