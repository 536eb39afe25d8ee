"""miniraytrace_b200 -- Python face of the B200 progressive path tracer.

Everything here is a thin ctypes layer over ``libmrt.so`` (the C ABI in
``include/mini_raytrace.h`` / ``include/mrt_ext.h``). ``Engine`` mirrors the
reference's C++ facade ``mrt::Engine`` (core/include/mrt/Engine.hpp:45-88):
scene edits, commit, render one frame, read the framebuffer.

There is no CPU fallback: if the library is missing ``load_library`` raises,
and if no suitable GPU is present ``Engine()`` raises ``MrtError`` with
``MRT_ERROR_VULKAN_INIT`` (the reference's device-initialisation code).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import abi
from .abi import *  # noqa: F401,F403  (re-export enums and structs)

# MRT_LIBRARY names another build of the library (the autotuner's variants)
_LIB_PATH = Path(os.environ.get("MRT_LIBRARY") or (Path(__file__).resolve().parent / "libmrt.so"))
_lib = None


class MrtError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        name = abi_result_name(code)
        super().__init__(f"{where}: {name} ({code}){': ' + detail if detail else ''}")


def abi_result_name(code: int) -> str:
    lib = load_library()
    return lib.mrtResultToString(code).decode()


def load_library(path: str | Path | None = None):
    """Load libmrt.so (built by ``python -m miniraytrace_b200.build``)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else _LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m miniraytrace_b200.build` "
                           "(there is no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, res, args in abi.FUNCTIONS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def last_error() -> str:
    return load_library().mrtGetLastErrorMessage().decode()


def _check(code: int, where: str):
    if code != abi.MRT_SUCCESS:
        raise MrtError(code, where, last_error())


def _f32(a, shape_last=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    return a


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f3(v):
    return abi.F3(*[float(x) for x in v])


def material_desc(base_color=(0.8, 0.8, 0.8), opacity=1.0, roughness=0.5, metallic=0.0, transmission=0.0,
                  ior=1.45, emission=(0.0, 0.0, 0.0), base_color_tex=0, roughness_tex=0, metallic_tex=0,
                  normal_tex=0, emission_tex=0) -> abi.MaterialDesc:
    """mrtMaterialDesc with the reference defaults (SceneTypes.hpp:80-94)."""
    return abi.MaterialDesc(baseColor=_f3(base_color), opacity=opacity, roughness=roughness, metallic=metallic,
                            transmission=transmission, ior=ior, emission=_f3(emission),
                            baseColorTex=base_color_tex, roughnessTex=roughness_tex, metallicTex=metallic_tex,
                            normalTex=normal_tex, emissionTex=emission_tex)


def light_desc(type=abi.MRT_LIGHT_SUN, direction=(0, 1, 0), position=(0, 0, 0), radiance=(1, 1, 1),
               angular_radius=0.00465, corner=(0, 0, 0), edge0=(1, 0, 0), edge1=(0, 0, 1),
               two_sided=False) -> abi.LightDesc:
    """mrtLightDesc with the reference defaults (SceneTypes.hpp:98-111)."""
    return abi.LightDesc(type=type, direction=_f3(direction), position=_f3(position), radiance=_f3(radiance),
                         angularRadius=angular_radius, corner=_f3(corner), edge0=_f3(edge0), edge1=_f3(edge1),
                         twoSided=1 if two_sided else 0)


def mesh_desc(positions, indices, normals=None, uvs=None):
    """Builds an mrtMeshDesc; returns (desc, keepalive arrays)."""
    pos = _f32(positions).reshape(-1, 3)
    idx = np.ascontiguousarray(np.asarray(indices, dtype=np.uint32)).reshape(-1)
    nrm = None if normals is None else _f32(normals).reshape(-1, 3)
    uv = None if uvs is None else _f32(uvs).reshape(-1, 2)
    d = abi.MeshDesc(vertexCount=pos.shape[0], indexCount=idx.size, positions=_ptr(pos), normals=_ptr(nrm),
                     uvs=_ptr(uv), indices=_ptr(idx))
    return d, (pos, idx, nrm, uv)


def texture_desc(pixels, fmt, generate_mips=False):
    """pixels: (H, W, 4) uint8 for RGBA8 formats, float32 for RGBA32F."""
    dt = np.float32 if fmt == abi.MRT_TEX_RGBA32F else np.uint8
    px = np.ascontiguousarray(np.asarray(pixels, dtype=dt))
    if px.ndim != 3 or px.shape[2] != 4:
        raise ValueError("texture pixels must be (H, W, 4)")
    d = abi.TextureDesc(width=px.shape[1], height=px.shape[0], format=fmt, pixels=_ptr(px),
                        generateMips=1 if generate_mips else 0)
    return d, px


def xform_rows(xf):
    """Row-major 3x4 transform as a float32 array of 12 (None stays None)."""
    if xf is None:
        return None
    a = _f32(xf).reshape(-1)
    if a.size == 16:
        a = a[:12]
    if a.size != 12:
        raise ValueError("transform must be 3x4 (or 4x4 with the last row dropped)")
    return np.ascontiguousarray(a)


class Engine:
    """One mrtEngine: a CUDA device, its scene and its accumulation buffers."""

    def __init__(self, width: int = 0, height: int = 0, gpu_index1: int = 0, validation: bool = False):
        self.lib = load_library()
        h = C.c_void_p()
        d = abi.EngineDesc(enableValidation=1 if validation else 0, width=width, height=height,
                           gpuIndex1=gpu_index1)
        _check(self.lib.mrtCreateEngine(C.byref(d), C.byref(h)), "mrtCreateEngine")
        self.h = h
        self.width = width or 1280
        self.height = height or 720

    # -- lifecycle
    def close(self):
        if getattr(self, "h", None):
            self.lib.mrtDestroyEngine(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- scene
    def add_mesh(self, positions, indices, normals=None, uvs=None) -> int:
        d, keep = mesh_desc(positions, indices, normals, uvs)
        return self.lib.mrtAddMesh(self.h, C.byref(d))

    def update_mesh(self, mesh_id, positions, indices, normals=None, uvs=None):
        d, keep = mesh_desc(positions, indices, normals, uvs)
        self.lib.mrtUpdateMesh(self.h, mesh_id, C.byref(d))

    def remove_mesh(self, mesh_id):
        self.lib.mrtRemoveMesh(self.h, mesh_id)

    def add_instance(self, mesh_id, xform=None, material=0) -> int:
        xf = xform_rows(xform)
        return self.lib.mrtAddInstance(self.h, mesh_id, _ptr(xf), material)

    def set_instance_transform(self, inst_id, xform):
        xf = xform_rows(xform)
        self.lib.mrtSetInstanceTransform(self.h, inst_id, _ptr(xf))

    def remove_instance(self, inst_id):
        self.lib.mrtRemoveInstance(self.h, inst_id)

    def add_material(self, desc: abi.MaterialDesc | None = None, **kw) -> int:
        d = desc if desc is not None else material_desc(**kw)
        return self.lib.mrtAddMaterial(self.h, C.byref(d))

    def update_material(self, mat_id, desc: abi.MaterialDesc | None = None, **kw):
        d = desc if desc is not None else material_desc(**kw)
        self.lib.mrtUpdateMaterial(self.h, mat_id, C.byref(d))

    def remove_material(self, mat_id):
        self.lib.mrtRemoveMaterial(self.h, mat_id)

    def add_texture(self, pixels, fmt=abi.MRT_TEX_RGBA8_SRGB, generate_mips=False) -> int:
        d, keep = texture_desc(pixels, fmt, generate_mips)
        return self.lib.mrtAddTexture(self.h, C.byref(d))

    def remove_texture(self, tex_id):
        self.lib.mrtRemoveTexture(self.h, tex_id)

    def add_light(self, desc: abi.LightDesc | None = None, **kw) -> int:
        d = desc if desc is not None else light_desc(**kw)
        return self.lib.mrtAddLight(self.h, C.byref(d))

    def update_light(self, light_id, desc: abi.LightDesc | None = None, **kw):
        d = desc if desc is not None else light_desc(**kw)
        self.lib.mrtUpdateLight(self.h, light_id, C.byref(d))

    def remove_light(self, light_id):
        self.lib.mrtRemoveLight(self.h, light_id)

    def set_environment(self, pixels, rotation=0.0, intensity=1.0):
        if pixels is None:
            self.lib.mrtSetEnvironment(self.h, None, 0.0, 0.0)
            return
        d, keep = texture_desc(pixels, abi.MRT_TEX_RGBA32F)
        self.lib.mrtSetEnvironment(self.h, C.byref(d), float(rotation), float(intensity))

    def set_camera(self, position=(0, 0, 5), target=(0, 0, 0), up=(0, 1, 0), fov_y_deg=45.0):
        d = abi.CameraDesc(position=_f3(position), target=_f3(target), up=_f3(up), fovYDeg=fov_y_deg)
        self.lib.mrtSetCamera(self.h, C.byref(d))

    def set_camera_ex(self, projection=abi.MRT_CAMERA_PERSPECTIVE, position=(0, 0, 5), forward=(0, 0, -1),
                      up=(0, 1, 0), left=-1.0, right=1.0, bottom=-1.0, top=1.0):
        d = abi.CameraDescEx(projection=projection, position=_f3(position), forward=_f3(forward), up=_f3(up),
                             left=left, right=right, bottom=bottom, top=top)
        self.lib.mrtSetCameraEx(self.h, C.byref(d))

    # -- commit / render
    def commit(self) -> dict:
        s = abi.CommitStats()
        _check(self.lib.mrtCommitScene(self.h, C.byref(s)), "mrtCommitScene")
        return {"blasRebuilt": s.blasRebuilt, "tlasRebuilt": bool(s.tlasRebuilt), "commitMs": s.commitMs}

    def set_render_settings(self, width=1280, height=720, max_bounces=8, spp_limit=1024, exposure_ev=0.0,
                            firefly_clamp=50.0, tonemap=abi.MRT_TONEMAP_ACES, denoise=True):
        d = abi.RenderSettings(width=width, height=height, maxBounces=max_bounces, sppLimit=spp_limit,
                               exposureEV=exposure_ev, fireflyClamp=firefly_clamp, tonemap=tonemap,
                               denoise=1 if denoise else 0)
        _check(self.lib.mrtSetRenderSettings(self.h, C.byref(d)), "mrtSetRenderSettings")
        self.width, self.height = width, height

    def render_frame(self) -> dict:
        fi = abi.FrameInfo()
        _check(self.lib.mrtRenderFrame(self.h, C.byref(fi)), "mrtRenderFrame")
        return {"spp": fi.spp, "converged": bool(fi.converged), "denoised": bool(fi.denoised),
                "frameMs": fi.frameMs}

    def render_frames(self, count: int) -> dict:
        fi = abi.FrameInfo()
        _check(self.lib.mrtxRenderFrames(self.h, count, C.byref(fi)), "mrtxRenderFrames")
        return {"spp": fi.spp, "converged": bool(fi.converged), "denoised": bool(fi.denoised),
                "frameMs": fi.frameMs}

    def read_framebuffer(self, fmt=abi.MRT_PIXEL_RGBA32F_LINEAR, out=None):
        if fmt == abi.MRT_PIXEL_RGBA32F_LINEAR:
            a = out if out is not None else np.empty((self.height, self.width, 4), np.float32)
        else:
            a = out if out is not None else np.empty((self.height, self.width, 4), np.uint8)
        _check(self.lib.mrtReadFramebuffer(self.h, fmt, a.ctypes.data_as(C.c_void_p), a.nbytes),
               "mrtReadFramebuffer")
        return a

    def reset_accumulation(self):
        self.lib.mrtResetAccumulation(self.h)

    # -- extensions
    def trace_rays(self, origins, dirs, t_max=1e30, wavefront=False):
        """Closest hits (mrtxTraceRays); wavefront=True traces them with the
        renderer's extend kernel (mrtxTraceRaysWavefront, tMax ignored)."""
        rays = make_rays(origins, dirs, t_max)
        hits = np.zeros(rays.shape[0], dtype=abi.HIT_DTYPE)
        fn = self.lib.mrtxTraceRaysWavefront if wavefront else self.lib.mrtxTraceRays
        _check(fn(self.h, _ptr(rays), rays.shape[0], _ptr(hits)), "mrtxTraceRays")
        return hits

    def trace_shadow_rays(self, origins, dirs, t_max=1e30):
        rays = make_rays(origins, dirs, t_max)
        occ = np.zeros(rays.shape[0], dtype=np.uint32)
        _check(self.lib.mrtxTraceShadowRays(self.h, _ptr(rays), rays.shape[0], _ptr(occ)), "mrtxTraceShadowRays")
        return occ

    def read_accumulation(self):
        a = np.empty((self.height, self.width, 4), np.float64)
        spp = C.c_uint32()
        _check(self.lib.mrtxReadAccumulation(self.h, _ptr(a), a.nbytes, C.byref(spp)), "mrtxReadAccumulation")
        return a, spp.value

    def stats(self) -> dict:
        s = abi.Stats()
        _check(self.lib.mrtxGetStats(self.h, C.byref(s)), "mrtxGetStats")
        return {k: getattr(s, k) for k, _ in abi.Stats._fields_ if k != "structSize"}

    def measure_l2_bandwidth(self) -> float:
        """L2 read bandwidth of this engine's GPU in GB/s (mrtxMeasureL2Bandwidth)."""
        g = C.c_float()
        _check(self.lib.mrtxMeasureL2Bandwidth(self.h, C.byref(g)), "mrtxMeasureL2Bandwidth")
        return g.value

    def build_env_cdf(self, rgba):
        px = np.ascontiguousarray(np.asarray(rgba, np.float32))
        h, w = px.shape[:2]
        cdf = np.empty(w * h + h, np.float32)
        integ = C.c_float()
        _check(self.lib.mrtxBuildEnvCdf(self.h, _ptr(px), w, h, _ptr(cdf), C.byref(integ)), "mrtxBuildEnvCdf")
        return cdf, integ.value

    def set_radiance_cache(self, enabled=True, training_paths=0, steps_per_sample=0, learning_rate=0.0, seed=1,
                           bounds=None, samples_per_update=0, training_vertices=0):
        """mrtxSetRadianceCache; bounds = (lo xyz, hi xyz) or None for the scene's."""
        d = abi.RadianceCacheDesc(enabled=1 if enabled else 0, trainingPaths=training_paths,
                                  stepsPerSample=steps_per_sample, learningRate=learning_rate, seed=seed,
                                  samplesPerUpdate=samples_per_update, trainingVertices=training_vertices)
        if bounds is not None:
            d.boundsLo[:] = [float(v) for v in bounds[0]]
            d.boundsHi[:] = [float(v) for v in bounds[1]]
        _check(self.lib.mrtxSetRadianceCache(self.h, C.byref(d)), "mrtxSetRadianceCache")

    def cache_query(self, features):
        f = np.ascontiguousarray(np.asarray(features, np.float32).reshape(-1, 16))
        out = np.empty((f.shape[0], 3), np.float32)
        _check(self.lib.mrtxRadianceCacheQuery(self.h, _ptr(f), f.shape[0], _ptr(out)), "mrtxRadianceCacheQuery")
        return out

    def cache_train(self, features, targets, steps=1):
        f = np.ascontiguousarray(np.asarray(features, np.float32).reshape(-1, 16))
        t = np.ascontiguousarray(np.asarray(targets, np.float32).reshape(-1, 3))
        loss = C.c_float()
        _check(self.lib.mrtxRadianceCacheTrain(self.h, _ptr(f), _ptr(t), f.shape[0], steps, C.byref(loss)),
               "mrtxRadianceCacheTrain")
        return loss.value

    def set_cache_averaging(self, decay: float):
        """mrtxSetRadianceCacheAveraging: moving-average decay of the weights
        queries read (0 = queries read the live weights)."""
        _check(self.lib.mrtxSetRadianceCacheAveraging(self.h, float(decay)), "mrtxSetRadianceCacheAveraging")

    def set_cache_schedule(self, lr_min: float, half_life_steps: float):
        """mrtxSetRadianceCacheSchedule: the training rate halves every
        half_life_steps Adam steps down to lr_min (0 = constant rate)."""
        _check(self.lib.mrtxSetRadianceCacheSchedule(self.h, float(lr_min), float(half_life_steps)),
               "mrtxSetRadianceCacheSchedule")

    def cache_gradients(self, features, targets):
        """mrtxRadianceCacheGradients: (grid gradient, MLP gradient, mean
        loss) of one batch, without an optimizer step."""
        f = np.ascontiguousarray(np.asarray(features, np.float32).reshape(-1, 16))
        t = np.ascontiguousarray(np.asarray(targets, np.float32).reshape(-1, 3))
        g = np.empty(abi.CACHE_GRID_FLOATS, np.float32)
        w = np.empty(abi.CACHE_MLP_FLOATS, np.float32)
        loss = C.c_float()
        _check(self.lib.mrtxRadianceCacheGradients(self.h, _ptr(f), _ptr(t), f.shape[0], _ptr(g), _ptr(w),
                                                   C.byref(loss)), "mrtxRadianceCacheGradients")
        return g, w, loss.value

    def set_denoiser(self, enabled=True, iterations=0, guide_samples=0, min_spp=0, sigma_color=0.0,
                     normal_power=0.0, sigma_albedo=0.0, sigma_depth=0.0):
        """mrtxSetDenoiser (zeros take the library's defaults)."""
        d = abi.DenoiserDesc(enabled=1 if enabled else 0, iterations=iterations, guideSamples=guide_samples,
                             minSpp=min_spp, sigmaColor=sigma_color, normalPower=normal_power,
                             sigmaAlbedo=sigma_albedo, sigmaDepth=sigma_depth)
        _check(self.lib.mrtxSetDenoiser(self.h, C.byref(d)), "mrtxSetDenoiser")

    def read_denoised(self):
        """mrtxReadDenoised: the denoised linear image (H x W x 4 float32)."""
        a = np.empty((self.height, self.width, 4), np.float32)
        _check(self.lib.mrtxReadDenoised(self.h, _ptr(a), a.nbytes), "mrtxReadDenoised")
        return a

    def read_denoiser_guides(self):
        """mrtxReadDenoiserGuides: (albedo, normal + distance), H x W x 4 float32 each."""
        al = np.empty((self.height, self.width, 4), np.float32)
        nd = np.empty((self.height, self.width, 4), np.float32)
        _check(self.lib.mrtxReadDenoiserGuides(self.h, _ptr(al), _ptr(nd), al.nbytes), "mrtxReadDenoiserGuides")
        return al, nd

    def cache_params(self, grid=None, mlp=None):
        """Returns (grid, mlp) as read, then writes the given arrays."""
        g = np.empty(abi.CACHE_GRID_FLOATS, np.float32)
        w = np.empty(abi.CACHE_MLP_FLOATS, np.float32)
        gi = None if grid is None else np.ascontiguousarray(np.asarray(grid, np.float32).ravel())
        wi = None if mlp is None else np.ascontiguousarray(np.asarray(mlp, np.float32).ravel())
        _check(self.lib.mrtxRadianceCacheParams(self.h, _ptr(g), _ptr(w), _ptr(gi), _ptr(wi)),
               "mrtxRadianceCacheParams")
        return g, w

    def set_sample_stream(self, offset: int, stride: int):
        _check(self.lib.mrtxSetSampleStream(self.h, offset, stride), "mrtxSetSampleStream")

    def set_traversal_budget(self, max_visits: int):
        """mrtxSetTraversalBudget: node visits per ray before the traversal
        gives up and the call fails (0 = the default, 2^22)."""
        _check(self.lib.mrtxSetTraversalBudget(self.h, max_visits), "mrtxSetTraversalBudget")

    def set_bvh_build_thresholds(self, min_triangles: int = 0, min_instances: int = 0):
        """mrtxSetBvhBuildThresholds: meshes of at least min_triangles
        triangles and instance sets of at least min_instances instances get
        their BVH built on the GPU, smaller ones on the host (0 = default;
        1 = always on the GPU; 0xFFFFFFFF = always on the host)."""
        _check(self.lib.mrtxSetBvhBuildThresholds(self.h, min_triangles, min_instances), "mrtxSetBvhBuildThresholds")

    def copy_accumulation_device(self, dev_ptr: int, nbytes: int, accumulate: bool):
        _check(self.lib.mrtxCopyAccumulationDevice(self.h, C.c_void_p(dev_ptr), nbytes, 1 if accumulate else 0),
               "mrtxCopyAccumulationDevice")


def build_env_cdf_no_alloc(dev_texels: int, width: int, height: int, dev_cdf: int, dev_integral: int,
                           stream: int = 0):
    """mrtxBuildEnvCdfNoAlloc over device pointers (integers): texels
    width*height RGBA32F, cdf width*height + height floats, integral one
    float, all on one GPU; stream a cudaStream_t handle (0 = legacy default
    stream). Asynchronous on that stream; allocates no device memory."""
    lib = load_library()
    _check(lib.mrtxBuildEnvCdfNoAlloc(C.c_void_p(dev_texels), width, height, C.c_void_p(dev_cdf),
                                      C.c_void_p(dev_integral), C.c_void_p(stream)), "mrtxBuildEnvCdfNoAlloc")


def inject_allocation_failure(succeed_first: int):
    """mrtxInjectAllocationFailure: the next `succeed_first` device or
    pinned-host allocations succeed, later ones fail as out of memory;
    a negative value turns the injection off."""
    _check(load_library().mrtxInjectAllocationFailure(succeed_first), "mrtxInjectAllocationFailure")


def render_batch(engines, spp):
    """mrtxRenderBatch: engines[i] renders spp[i] more samples; all engines'
    waves are issued before any is waited for. Returns each engine's frame
    info (spp, converged, frameMs = call start to that engine's completion)."""
    lib = load_library()
    n = len(engines)
    handles = (C.c_void_p * n)(*[e.h for e in engines])
    counts = (C.c_uint32 * n)(*[int(k) for k in spp])
    infos = (abi.FrameInfo * n)()
    for i in range(n):
        infos[i].structSize = C.sizeof(abi.FrameInfo)
    _check(lib.mrtxRenderBatch(handles, counts, n, infos), "mrtxRenderBatch")
    return [dict(spp=infos[i].spp, converged=bool(infos[i].converged), frameMs=infos[i].frameMs) for i in range(n)]


def build_mesh_bvh(positions, indices, builder=abi.MRTX_BVH_HOST_SAH, max_leaf_prims=3, engine=None):
    """The engine's 8-wide BVH of a triangle mesh from one builder
    (abi.MRTX_BVH_*): (nodes as a WIDE_NODE_DTYPE array, triangle order).
    The device builder needs an Engine."""
    lib = load_library()
    p = np.ascontiguousarray(np.asarray(positions, np.float32).reshape(-1, 3))
    i = np.ascontiguousarray(np.asarray(indices, np.uint32).reshape(-1, 3))
    nt = i.shape[0]
    cap = max(1, nt)
    nodes = np.zeros(cap, dtype=abi.WIDE_NODE_DTYPE)
    order = np.zeros(max(1, nt), np.uint32)
    count = C.c_uint32()
    handle = engine.h if engine is not None else None
    _check(lib.mrtxBuildMeshBvh(handle, _ptr(p), p.shape[0], _ptr(i), nt, builder, max_leaf_prims, _ptr(nodes), cap,
                                _ptr(order), C.byref(count)), "mrtxBuildMeshBvh")
    return nodes[:count.value].copy(), order[:nt].copy()


def build_wide_bvh(aabbs, max_leaf_prims=3):
    """Host build of the engine's 8-wide BVH over (N, 6) boxes:
    (nodes as a WIDE_NODE_DTYPE array, primitive order)."""
    lib = load_library()
    a = np.ascontiguousarray(np.asarray(aabbs, np.float32).reshape(-1, 6))
    n = a.shape[0]
    cap = max(1, n)
    nodes = np.zeros(cap, dtype=abi.WIDE_NODE_DTYPE)
    order = np.zeros(max(1, n), np.uint32)
    count = C.c_uint32()
    _check(lib.mrtxBuildWideBvh(_ptr(a), n, max_leaf_prims, _ptr(nodes), cap, _ptr(order), C.byref(count)),
           "mrtxBuildWideBvh")
    return nodes[:count.value].copy(), order[:n].copy()


def make_rays(origins, dirs, t_max=1e30):
    o = np.asarray(origins, np.float32).reshape(-1, 3)
    d = np.asarray(dirs, np.float32).reshape(-1, 3)
    rays = np.zeros(o.shape[0], dtype=abi.RAY_DTYPE)
    rays["origin"] = o
    rays["dir"] = d
    rays["tMax"] = t_max
    return rays
