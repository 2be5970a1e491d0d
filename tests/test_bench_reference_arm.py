"""The reference arm of bench.py (the reference's CPU hydro on the host
cores) prints one JSON line with the C1 line's metric, unit and config, the
`impl`, `cpu_baseline` and `e2e` keys, on a bounded sample."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line(tmp_path):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    if "unavailable" in line:
        return
    sys.path.insert(0, ROOT)
    import bench
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["higher_is_better"] is True and line["steps"] == 1
    # the C1 config's keys, with the workload naming the sample that ran
    full = bench.c1_config((256, 256, 256), 1)
    assert set(line["config"]) == set(full)
    assert line["config"]["workload"].startswith("c1 sample: 128^3")
    assert line["config"]["domain"] == [128, 128, 128]
    assert line["value"] > 0 and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"],
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
