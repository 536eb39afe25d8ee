"""Host-side scene store checks (no GPU): tests/host/scene_store_check.cpp
compiled with g++ against csrc/host/scene.cpp and run; see that file for
what it checks (threaded mesh copies and index checks, lazy tangents)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_scene_store_host_checks(tmp_path):
    exe = tmp_path / "scene_store_check"
    host = ROOT / "miniraytrace_b200" / "csrc" / "host"
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-pthread", "-I", str(host), "-I", str(ROOT / "include"),
           str(ROOT / "tests" / "host" / "scene_store_check.cpp"), str(host / "scene.cpp"), "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
