"""bench.py's reference arm (--impl reference) runs on the host alone: one
JSON line with the contract's keys, on a small grid so that it stays quick."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--grid", "12",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["steps"] == 2 and line["value"] > 0
    # the steps that ran are timed whole: steps x ms_per_step is the time they took
    assert line["ms_per_step"] > 0 and line["spai_seconds_per_build"] * 1e3 <= line["ms_per_step"]
    assert line["pcg_status"] == 1
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["grid"] == 12 and line["config"]["n"] == 12 ** 3


def test_reference_arm_caps_its_steps():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--grid", "10",
                          "--steps", "9", "--warmup", "5"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["steps"] == 3 and line["warmup"] == 1
    assert line["steps_requested"] == 9 and line["warmup_requested"] == 5
