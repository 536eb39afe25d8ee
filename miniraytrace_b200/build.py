"""Build libmrt.so in-tree: CUDA kernels for sm_100a (nvcc) + host C++ (g++).

Usage: ``python -m miniraytrace_b200.build [--force]``.

The result, ``miniraytrace_b200/libmrt.so``, links the CUDA runtime statically
and exports only the ``mrt*`` C ABI (every other symbol is hidden), so a
caller needs nothing but the NVIDIA driver. Objects go to
``miniraytrace_b200/_build/`` and are rebuilt when their source or any header
under ``csrc/`` or ``include/`` is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libmrt.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-I", str(CSRC), "-I", str(ROOT / "include"),
]
# Per-file extra nvcc flags. The path-tracing translation unit is compiled
# without multiply-add contraction so its shading arithmetic is the same
# sequence of IEEE single-precision operations as the CPU evaluation (explicit
# __fmaf_rn intrinsics still produce fused multiply-adds where wanted).
NVCC_FILE_FLAGS = {"pathtrace.cu": ["-fmad=false"], "bvh_build.cu": ["-fmad=false"]}

CXX_FLAGS = [
    "-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-ffp-contract=off",
    "-Wall", "-Wextra", "-Wno-unused-parameter",
    "-I", str(CUDA_HOME / "include"), "-I", str(CSRC), "-I", str(ROOT / "include"),
]


def _sources():
    cu = sorted((CSRC / "cuda").glob("*.cu"))
    cpp = sorted((CSRC / "host").glob("*.cpp"))
    return cu, cpp


def _headers_mtime() -> float:
    hs = list(CSRC.rglob("*.h")) + list(CSRC.rglob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _stale(obj: Path, src: Path, hdr: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return t < src.stat().st_mtime or t < hdr


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every kernel for sm_100a and link libmrt.so. Returns its path."""
    if not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    BUILD.mkdir(exist_ok=True)
    cu, cpp = _sources()
    hdr = _headers_mtime()
    jobs = []
    objs = []
    for src in cu:
        obj = BUILD / (src.stem + ".cu.o")
        objs.append(obj)
        if force or _stale(obj, src, hdr):
            jobs.append([NVCC, *NVCC_FLAGS, *NVCC_FILE_FLAGS.get(src.name, []), "-c", str(src), "-o", str(obj)])
    for src in cpp:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src, hdr):
            jobs.append(["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as ex:
            for r in ex.map(_run, jobs):
                if verbose and r.stderr:
                    sys.stderr.write(r.stderr)
    relink = force or bool(jobs) or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs)
    if relink:
        tmp = BUILD / "libmrt.so.tmp"
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs),
              "-Xlinker", "--exclude-libs,ALL", "-Xlinker", "-z,defs",
              "-Xlinker", f"--version-script={CSRC / 'exports.map'}", "-lpthread", "-ldl", "-lrt"])
        shutil.move(str(tmp), str(LIB))
    return LIB


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose=True)
    print(p)
