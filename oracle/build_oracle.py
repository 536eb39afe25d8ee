"""ORACLE -- test infrastructure only.

Builds the CPU oracle (``oracle/_build/liboracle.so``, from the restatement in
this directory) and, when the reference checkout is present, three libraries
of the reference's own code compiled from its sources where they lie
(nothing is copied into this repository; outputs go to the git-ignored
``oracle/_ref/``), against the glm-subset shim in ``oracle/glm_shim``:

- ``libref_bvh.so``: ``core/src/accel/Bvh.cpp`` (the binned-SAH builder);
- ``libref_scene.so``: ``core/src/scene/Scene.cpp`` (the scene store with its
  derived normals and tangents, Scene.cpp:13-60);
- ``libref_envcdf.so``: the environment-CDF loop of ``Renderer::packEnvironment``
  (core/src/render/Renderer.cpp:620-655). Renderer.cpp as a whole needs the
  Vulkan headers and generated SPIR-V, so the recipe compiles only that loop:
  at build time it takes the statements from ``std::vector<float> cdf(`` to
  the ``m_envIntegral =`` assignment out of the reference file into a
  generated source under ``oracle/_ref/`` (``#line`` points back at the
  reference file), inside a function whose parameters carry the loop's
  inputs (``px``, ``w``, ``h``).

The reference checkout is found at ``--reference PATH``, else the
``MRT_REFERENCE_DIR`` environment variable, else ``/root/reference``. Without
it only the oracle is built (the GPU box runs the prebuilt ``oracle/_ref``
libraries that travel with the tree, if any).

Everything is compiled with ``-ffp-contract=off`` so FP32 arithmetic is plain
IEEE single precision, as the reference shaders specify it. (The reference's
own host build may contract multiply-adds; that is not reproducible here.)
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
DEFAULT_REF = Path("/root/reference")
OUT = HERE / "_build" / "liboracle.so"
REF_DIR = HERE / "_ref"
REF_OUT = REF_DIR / "libref_bvh.so"
REF_SCENE_OUT = REF_DIR / "libref_scene.so"
REF_ENVCDF_OUT = REF_DIR / "libref_envcdf.so"
FLAGS = ["-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math"]
ENV_CDF_FIRST = "std::vector<float> cdf(size_t(w) * h + h);"
ENV_CDF_LAST = "m_envIntegral ="


def reference_dir(path: str | Path | None = None) -> Path:
    return Path(path or os.environ.get("MRT_REFERENCE_DIR") or DEFAULT_REF)


def _newer(out: Path, srcs) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(s).stat().st_mtime > t for s in srcs)


def _compile(out: Path, args, force: bool, deps) -> None:
    if not (force or _newer(out, deps)):
        return
    out.parent.mkdir(exist_ok=True)
    tmp = out.with_suffix(".tmp")
    subprocess.run(["g++", *FLAGS, "-std=c++20", "-I", str(HERE / "glm_shim"), *args, "-o", str(tmp)], check=True)
    tmp.replace(out)


def env_cdf_source(renderer_cpp: Path) -> str:
    """The generated translation unit around the reference's CDF loop."""
    lines = renderer_cpp.read_text().splitlines()
    first = next(i for i, ln in enumerate(lines) if ENV_CDF_FIRST in ln)
    last = next(i for i in range(first, len(lines)) if ENV_CDF_LAST in lines[i])
    body = "\n".join(lines[first:last + 1])
    return f"""// Generated by oracle/build_oracle.py: the statements of
// {renderer_cpp.name}:{first + 1}-{last + 1} compiled as they are, inside a function whose
// parameters and locals stand for the Renderer members the loop reads and writes.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <glm/glm.hpp>

extern "C" void ref_env_cdf(const float* px, uint32_t w, uint32_t h, float* cdfOut, float* integralOut) {{
    uint32_t m_envCdfW = 0, m_envCdfH = 0;
    float m_envIntegral = 0.0f;
#line {first + 1} "{renderer_cpp}"
{body}
    (void)m_envCdfW;
    (void)m_envCdfH;
    std::memcpy(cdfOut, cdf.data(), cdf.size() * sizeof(float));
    *integralOut = m_envIntegral;
}}
"""


def build(force: bool = False, reference: str | Path | None = None) -> Path:
    srcs = sorted(HERE.glob("*.hpp")) + [HERE / "oracle_capi.cpp", HERE.parent / "include" / "mini_raytrace.h"]
    if force or _newer(OUT, srcs):
        OUT.parent.mkdir(exist_ok=True)
        tmp = OUT.with_suffix(".tmp")
        subprocess.run(["g++", *FLAGS, "-o", str(tmp), str(HERE / "oracle_capi.cpp"), "-lpthread"], check=True)
        tmp.replace(OUT)
    ref = reference_dir(reference)
    shim = HERE / "glm_shim" / "glm" / "glm.hpp"
    inc = ["-I", str(ref / "core" / "include")]
    bvh_cpp = ref / "core" / "src" / "accel" / "Bvh.cpp"
    if bvh_cpp.exists():
        _compile(REF_OUT, [*inc, "-I", str(bvh_cpp.parent), str(HERE / "ref_bvh_wrap.cpp"), str(bvh_cpp)], force,
                 [bvh_cpp, HERE / "ref_bvh_wrap.cpp", shim])
    scene_cpp = ref / "core" / "src" / "scene" / "Scene.cpp"
    if scene_cpp.exists():
        _compile(REF_SCENE_OUT, [*inc, str(HERE / "ref_scene_wrap.cpp"), str(scene_cpp)], force,
                 [scene_cpp, HERE / "ref_scene_wrap.cpp", shim])
    renderer_cpp = ref / "core" / "src" / "render" / "Renderer.cpp"
    if renderer_cpp.exists():
        gen = REF_DIR / "ref_env_cdf_gen.cpp"
        if force or _newer(REF_ENVCDF_OUT, [renderer_cpp, shim, Path(__file__)]):
            REF_DIR.mkdir(exist_ok=True)
            gen.write_text(env_cdf_source(renderer_cpp))
        _compile(REF_ENVCDF_OUT, [str(gen)], force, [gen, shim])
    return OUT


if __name__ == "__main__":
    ref_arg = None
    if "--reference" in sys.argv:
        ref_arg = sys.argv[sys.argv.index("--reference") + 1]
    print(build(force="--force" in sys.argv, reference=ref_arg))
