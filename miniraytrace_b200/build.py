"""Build libmrt.so in-tree: CUDA kernels for sm_100a (nvcc) + host C++ (g++).

Usage: ``python -m miniraytrace_b200.build [--force]``.

The result, ``miniraytrace_b200/libmrt.so``, links the CUDA runtime statically
and exports only the ``mrt*`` C ABI (every other symbol is hidden), so a
caller needs nothing but the NVIDIA driver. Objects go to
``miniraytrace_b200/_build/`` and are rebuilt when their source or any header
under ``csrc/`` or ``include/`` is newer, or when the kernels' tunable
constants change.

Tunable constants (thread-block sizes, register bounds, traversal
scheduling thresholds) are preprocessor defines of the CUDA sources. Their
values come from ``miniraytrace_b200/tuned.json``, written by the autotuner
(``python -m miniraytrace_b200.autotune``); a define missing there keeps
the default in the source. ``build(defines=..., lib=..., build_dir=...)``
builds a variant elsewhere, which is how the autotuner measures candidates.
"""
from __future__ import annotations

import concurrent.futures as cf
import fcntl
import json
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
TUNED = PKG / "tuned.json"
# Sources that read the tunable defines; a variant rebuilds only these and
# links them with the shared objects of the main build directory.
TUNED_SOURCES = {"pathtrace.cu"}

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


def tuned_defines() -> dict:
    """The kernels' tunable constants chosen by the autotuner (name -> value)."""
    if TUNED.exists():
        return dict(json.loads(TUNED.read_text()).get("defines", {}))
    return {}


def build(force: bool = False, verbose: bool = False, defines: dict | None = None, lib: Path | None = None,
          build_dir: Path | None = None) -> Path:
    """Compile every kernel for sm_100a and link libmrt.so. Returns its path.
    defines: the tunable constants (default: tuned.json); lib / build_dir:
    where a variant goes (default: the package's libmrt.so and _build/)."""
    if lib is None and os.environ.get("MRT_LIBRARY"):
        return Path(os.environ["MRT_LIBRARY"])  # a variant built by its own build() call
    if not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    defines = tuned_defines() if defines is None else dict(defines)
    out = Path(lib) if lib else LIB
    bdir = Path(build_dir) if build_dir else BUILD
    bdir.mkdir(parents=True, exist_ok=True)
    BUILD.mkdir(exist_ok=True)
    # one build at a time: the ranks of a multi-GPU run (and parallel test
    # workers) call build() together; the first compiles, the others wait
    # for its lock and then find every object fresh
    with open(BUILD / ".build.lock", "w") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        try:
            return _build_locked(force, verbose, defines, out, bdir)
        finally:
            fcntl.flock(lock, fcntl.LOCK_UN)


def _build_locked(force, verbose, defines, out, bdir) -> Path:
    dflags = [f"-D{k}={v}" for k, v in sorted(defines.items())]
    stamp = bdir / "defines.txt"
    retune = not stamp.exists() or stamp.read_text() != " ".join(dflags)
    cu, cpp = _sources()
    hdr = _headers_mtime()
    jobs = []
    objs = []
    for src in cu:
        tuned = src.name in TUNED_SOURCES
        obj = (bdir if tuned else BUILD) / (src.stem + ".cu.o")
        objs.append(obj)
        if force or (tuned and retune) or _stale(obj, src, hdr):
            jobs.append([NVCC, *NVCC_FLAGS, *(dflags if tuned else []), *NVCC_FILE_FLAGS.get(src.name, []), "-c",
                         str(src), "-o", str(obj)])
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
    stamp.write_text(" ".join(dflags))
    relink = force or bool(jobs) or not out.exists() or out.stat().st_mtime < max(o.stat().st_mtime for o in objs)
    if relink:
        tmp = bdir / "libmrt.so.tmp"
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs),
              "-Xlinker", "--exclude-libs,ALL", "-Xlinker", "-z,defs",
              "-Xlinker", f"--version-script={CSRC / 'exports.map'}", "-lpthread", "-ldl", "-lrt"])
        shutil.move(str(tmp), str(out))
    return out


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose=True)
    print(p)
