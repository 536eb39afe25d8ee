"""CPU checks of the drop-in boundary: libmrt.so loads, exports exactly the
symbols declared in include/*.h, the ctypes layouts equal the C layouts, and
the argument/handle rules of the reference translation layer hold without a
device (reference capi/src/capi.cpp:22-316)."""
import ctypes as C
import re
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from conftest import gpu_available

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        for m in re.finditer(r"MRT_API\s+[\w\s\*]+?\b(mrt\w+)\s*\(", h.read_text()):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported(mrt_lib):
    names = declared_functions()
    assert len(names) >= 27 + 8
    out = subprocess.run(["nm", "-D", "--defined-only", str(mrt_lib._LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert names <= exported
    assert exported == names, f"unexpected exports: {sorted(exported - names)}"
    lib = mrt_lib.load_library()
    for n in names:
        assert getattr(lib, n)


def test_reference_abi_function_set(mrt_lib):
    """The 27 functions of reference capi/include/mini_raytrace.h:184-237."""
    ref = {"mrtCreateEngine", "mrtDestroyEngine", "mrtAddMesh", "mrtUpdateMesh", "mrtRemoveMesh",
           "mrtAddInstance", "mrtSetInstanceTransform", "mrtRemoveInstance", "mrtAddMaterial",
           "mrtUpdateMaterial", "mrtRemoveMaterial", "mrtAddTexture", "mrtRemoveTexture", "mrtAddLight",
           "mrtUpdateLight", "mrtRemoveLight", "mrtSetEnvironment", "mrtSetCamera", "mrtSetCameraEx",
           "mrtCommitScene", "mrtSetRenderSettings", "mrtRenderFrame", "mrtReadFramebuffer",
           "mrtResetAccumulation", "mrtSetLogCallback", "mrtResultToString", "mrtGetLastErrorMessage"}
    assert len(ref) == 27
    assert ref <= declared_functions()


STRUCTS = ["mrtEngineDesc", "mrtMeshDesc", "mrtMaterialDesc", "mrtTextureDesc", "mrtLightDesc", "mrtCameraDesc",
           "mrtCameraDescEx", "mrtRenderSettings", "mrtFrameInfo", "mrtCommitStats", "mrtxRay", "mrtxHit",
           "mrtxStats", "mrtxRadianceCacheDesc", "mrtxDenoiserDesc"]


def test_ctypes_layouts_match_c(mrt_lib):
    from miniraytrace_b200 import abi
    py = {"mrtEngineDesc": abi.EngineDesc, "mrtMeshDesc": abi.MeshDesc, "mrtMaterialDesc": abi.MaterialDesc,
          "mrtTextureDesc": abi.TextureDesc, "mrtLightDesc": abi.LightDesc, "mrtCameraDesc": abi.CameraDesc,
          "mrtCameraDescEx": abi.CameraDescEx, "mrtRenderSettings": abi.RenderSettings,
          "mrtFrameInfo": abi.FrameInfo, "mrtCommitStats": abi.CommitStats, "mrtxRay": abi.Ray,
          "mrtxHit": abi.Hit, "mrtxStats": abi.Stats, "mrtxRadianceCacheDesc": abi.RadianceCacheDesc,
          "mrtxDenoiserDesc": abi.DenoiserDesc}
    src = '#include <stdio.h>\n#include <stddef.h>\n#include "mrt_ext.h"\nint main(void){\n'
    for s in STRUCTS:
        src += f'printf("{s} %zu\\n", sizeof({s}));\n'
        for f, _ in py[s]._fields_:
            src += f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));\n'
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as td:
        c = Path(td) / "l.c"
        c.write_text(src)
        exe = Path(td) / "l"
        subprocess.run(["gcc", "-I", str(ROOT / "include"), str(c), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    vals = dict(line.rsplit(" ", 1) for line in out.splitlines())
    for s in STRUCTS:
        assert int(vals[s]) == C.sizeof(py[s]), s
        for f, _ in py[s]._fields_:
            assert int(vals[f"{s}.{f}"]) == getattr(py[s], f).offset, f"{s}.{f}"
    # reference C# smoke test size checks (rhino/MiniRaytrace.Smoke/Program.cs:30-33)
    assert C.sizeof(abi.CameraDescEx) == 8 + 4 + 12 * 3 + 4 * 4
    assert C.sizeof(abi.Ray) == 32 and C.sizeof(abi.Hit) == 32


def test_enum_values(mrt_lib):
    from miniraytrace_b200 import abi
    assert (abi.MRT_SUCCESS, abi.MRT_ERROR_UNKNOWN, abi.MRT_ERROR_VULKAN_INIT, abi.MRT_ERROR_OUT_OF_MEMORY,
            abi.MRT_ERROR_INVALID_ARGUMENT, abi.MRT_ERROR_INVALID_HANDLE, abi.MRT_ERROR_SHADER_LOAD,
            abi.MRT_ERROR_DEVICE_LOST) == tuple(range(8))
    lib = mrt_lib.load_library()
    names = [lib.mrtResultToString(i).decode() for i in range(8)]
    assert names == ["Success", "ErrorUnknown", "ErrorVulkanInit", "ErrorOutOfMemory", "ErrorInvalidArgument",
                     "ErrorInvalidHandle", "ErrorShaderLoad", "ErrorDeviceLost"]
    assert lib.mrtResultToString(99).decode() == "ErrorUnknown"


def test_null_and_short_struct_handling(mrt_lib):
    from miniraytrace_b200 import abi
    lib = mrt_lib.load_library()
    h = C.c_void_p()
    assert lib.mrtCreateEngine(None, C.byref(h)) == abi.MRT_ERROR_INVALID_ARGUMENT
    d = abi.EngineDesc()
    assert lib.mrtCreateEngine(C.byref(d), None) == abi.MRT_ERROR_INVALID_ARGUMENT
    short = abi.EngineDesc()
    short.structSize = 8
    assert lib.mrtCreateEngine(C.byref(short), C.byref(h)) == abi.MRT_ERROR_INVALID_ARGUMENT
    assert lib.mrtCommitScene(None, None) == abi.MRT_ERROR_INVALID_HANDLE
    assert lib.mrtRenderFrame(None, None) == abi.MRT_ERROR_INVALID_HANDLE
    buf = np.zeros(16, np.float32)
    assert lib.mrtReadFramebuffer(None, 1, buf.ctypes.data_as(C.c_void_p), 64) == abi.MRT_ERROR_INVALID_ARGUMENT
    rs = abi.RenderSettings(width=8, height=8)
    assert lib.mrtSetRenderSettings(None, C.byref(rs)) == abi.MRT_ERROR_INVALID_ARGUMENT
    md = abi.MeshDesc()
    assert lib.mrtAddMesh(None, C.byref(md)) == abi.MRT_INVALID_ID
    assert lib.mrtAddInstance(None, 1, None, 0) == abi.MRT_INVALID_ID
    assert lib.mrtAddMaterial(None, None) == abi.MRT_INVALID_ID
    assert lib.mrtAddLight(None, None) == abi.MRT_INVALID_ID
    assert lib.mrtAddTexture(None, None) == abi.MRT_INVALID_ID
    lib.mrtDestroyEngine(None)  # safe
    lib.mrtRemoveMesh(None, 1)
    lib.mrtSetEnvironment(None, None, 0.0, 1.0)
    lib.mrtResetAccumulation(None)
    assert lib.mrtxRenderFrames(None, 1, None) == abi.MRT_ERROR_INVALID_HANDLE
    assert lib.mrtxTraceRays(None, None, 0, None) == abi.MRT_ERROR_INVALID_HANDLE
    assert lib.mrtxReadAccumulation(None, None, 0, None) == abi.MRT_ERROR_INVALID_HANDLE
    assert lib.mrtxMeasureL2Bandwidth(None, None) == abi.MRT_ERROR_INVALID_HANDLE
    assert lib.mrtxGetStats(None, None) == abi.MRT_ERROR_INVALID_HANDLE
    assert lib.mrtxSetBvhBuildThresholds(None, 1, 1) == abi.MRT_ERROR_INVALID_HANDLE
    assert lib.mrtxSetTraversalBudget(None, 1) == abi.MRT_ERROR_INVALID_HANDLE
    assert lib.mrtGetLastErrorMessage() is not None


def test_log_callback_roundtrip(mrt_lib):
    from miniraytrace_b200 import abi
    lib = mrt_lib.load_library()
    seen = []
    cb = abi.LOG_FN(lambda level, msg, user: seen.append((level, msg.decode())))
    lib.mrtSetLogCallback(cb, None)
    try:
        if not gpu_available():
            h = C.c_void_p()
            d = abi.EngineDesc(width=8, height=8)
            assert lib.mrtCreateEngine(C.byref(d), C.byref(h)) == abi.MRT_ERROR_VULKAN_INIT
            assert any(level == 3 for level, _ in seen)
    finally:
        lib.mrtSetLogCallback(abi.LOG_FN(), None)


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_create_engine_without_device_fails_cleanly(mrt_lib):
    from miniraytrace_b200 import MrtError, abi
    with pytest.raises(MrtError) as e:
        mrt_lib.Engine(16, 16)
    assert e.value.code == abi.MRT_ERROR_VULKAN_INIT
    assert "CUDA" in mrt_lib.last_error()
