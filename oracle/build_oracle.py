"""ORACLE -- test infrastructure only.

Builds the CPU oracle (``oracle/_build/liboracle.so``, from the restatement in
this directory) and, when the reference checkout is present at
``/root/reference``, the reference's own BVH builder
(``oracle/_ref/libref_bvh.so`` from ``core/src/accel/Bvh.cpp`` compiled in
place, against the glm-subset shim in ``oracle/glm_shim``). The reference's
sources are read where they lie; nothing is copied into this repository.

The oracle is compiled with ``-ffp-contract=off`` so FP32 arithmetic is plain
IEEE single precision, as the reference shaders specify it.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF = Path("/root/reference")
OUT = HERE / "_build" / "liboracle.so"
REF_OUT = HERE / "_ref" / "libref_bvh.so"
FLAGS = ["-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math"]


def _newer(out: Path, srcs) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(s).stat().st_mtime > t for s in srcs)


def build(force: bool = False) -> Path:
    srcs = sorted(HERE.glob("*.hpp")) + [HERE / "oracle_capi.cpp", HERE.parent / "include" / "mini_raytrace.h"]
    if force or _newer(OUT, srcs):
        OUT.parent.mkdir(exist_ok=True)
        tmp = OUT.with_suffix(".tmp")
        subprocess.run(["g++", *FLAGS, "-o", str(tmp), str(HERE / "oracle_capi.cpp"), "-lpthread"], check=True)
        tmp.replace(OUT)
    bvh_cpp = REF / "core" / "src" / "accel" / "Bvh.cpp"
    if bvh_cpp.exists():
        rsrcs = [bvh_cpp, HERE / "ref_bvh_wrap.cpp", HERE / "glm_shim" / "glm" / "glm.hpp"]
        if force or _newer(REF_OUT, rsrcs):
            REF_OUT.parent.mkdir(exist_ok=True)
            tmp = REF_OUT.with_suffix(".tmp")
            subprocess.run(["g++", *FLAGS, "-std=c++20", "-I", str(HERE / "glm_shim"),
                            "-I", str(REF / "core" / "include"), "-I", str(REF / "core" / "src" / "accel"),
                            "-o", str(tmp), str(HERE / "ref_bvh_wrap.cpp"), str(bvh_cpp)], check=True)
            tmp.replace(REF_OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
