"""bench.py's reference arm, which runs on the host cores: its JSON line
carries the fields the measurement contract names, GPU-only modes print one
`unavailable` line and exit 0, and ranks other than 0 exit 0 silently."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def run_bench(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT, env=e, capture_output=True,
                       text=True, timeout=600)
    return r.returncode, [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_reference_arm_line(oracle_lib):
    rc, lines = run_bench("--impl", "reference", "--config", "box_sphere", "--steps", "2", "--warmup", "3",
                          "--cpu-seconds", "2")
    assert rc == 0 and len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]


def test_gpu_only_modes_print_unavailable():
    for mode in ("room", "cache", "batch", "large"):
        rc, lines = run_bench("--impl", "reference", "--config", mode)
        assert rc == 0 and len(lines) == 1
        d = json.loads(lines[0])
        assert d["impl"] == "reference" and mode in d["unavailable"]


def test_reference_arm_other_ranks_exit_silently():
    rc, lines = run_bench("--impl", "reference", "--config", "box_sphere", env={"RANK": "1", "WORLD_SIZE": "2"})
    assert rc == 0 and lines == []
