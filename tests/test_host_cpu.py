"""Host-side checks without a GPU: C++ harnesses under tests/host/ compiled
with g++ against the library's host sources and run. scene_store_check.cpp:
the scene store (threaded mesh copies and index checks, lazy tangents);
copy_pool_check.cpp: the threaded copy behind readback and staged uploads."""
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


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_copy_pool_host_checks(tmp_path):
    exe = tmp_path / "copy_pool_check"
    host = ROOT / "miniraytrace_b200" / "csrc" / "host"
    cmd = ["g++", "-O2", "-std=c++17", "-pthread", "-I", str(host), str(ROOT / "tests" / "host" / "copy_pool_check.cpp"),
           str(host / "copy_pool.cpp"), "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr

