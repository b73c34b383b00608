"""bench.py's output contract, checked on the CPU: the reference arm's JSON
line (the CPU oracle on a tiny sample) carries every key the harness reads,
and the argument parser accepts the documented options."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line_has_the_contract_keys():
    out = subprocess.run(
        [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
         "--warmup", "3", "--ref-sample", "12", "--no-ref-gpu-chem"],
        capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference"
    assert line["metric"] == "cell-updates/s (256^3 Euler)" and line["unit"] == "cell-updates/s"
    assert line["value"] > 0.0 and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["warmup"] == 3
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] == "port" and cb["cores"] >= 1
    e2e = line["e2e"]
    assert e2e["value"] == line["value"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert "workload" in line["config"]
    # the line describes what it timed: a 12^3 block, whose measured step time
    # gives the value
    assert line["config"]["cells"] == 12 ** 3
    assert line["config"]["same_config_as_ours"] is False
    assert abs(line["ms_per_step"] * 1e-3 * line["value"] / 12 ** 3 - 1.0) < 1e-9


def test_bench_options_parse():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0
    for opt in ("--gpus", "--steps", "--warmup", "--impl", "--precision", "--tile", "--part",
                "--headline-only", "--no-ref-gpu-chem", "--curv-n"):
        assert opt in out.stdout, opt
