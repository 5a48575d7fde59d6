"""bench.py's reference arm on the CPU: one warm-up and one timed step of the
CPU oracle on the 128^3 plume, printed as one JSON line in the bench format
with the same config object as our arm's line."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_bench_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["unit"] == "Mcell-steps/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1 and line["n_gpus"] == 1
    assert line["warmup"] == 1
    sys.path.insert(0, ROOT)
    import bench
    assert line["config"] == bench.bench_config("fp64_cg", 128, 1)
    assert line["config"]["grid"] == [128, 128, 128] and line["config"]["form"] == "fp64_cg"
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] == 1 and cb["value"] == line["value"]
    assert "CG iters [200]" in cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"],
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
