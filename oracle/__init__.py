"""ORACLE -- test infrastructure only. Not part of the product.

ctypes face of the CPU restatement of the MiniRaytrace shader math
(liboracle.so, built by ``oracle/build_oracle.py``) and of the reference's own
code compiled from its sources into ``oracle/_ref/``: the BVH builder
(``libref_bvh.so``), the scene store's derived normals and tangents
(``libref_scene.so``) and the environment-CDF loop (``libref_envcdf.so``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this package, and only as the checker / the CPU baseline.
``OracleScene`` exposes the same scene-building methods as
``miniraytrace_b200.Engine`` so one scene description drives both.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from miniraytrace_b200 import abi
from miniraytrace_b200 import light_desc, material_desc, mesh_desc, texture_desc, xform_rows

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
REF_BVH_PATH = HERE / "_ref" / "libref_bvh.so"
REF_SCENE_PATH = HERE / "_ref" / "libref_scene.so"
REF_ENVCDF_PATH = HERE / "_ref" / "libref_envcdf.so"

_lib = None
_ref = None
_ref_scene = None
_ref_envcdf = None

NODE_DTYPE = np.dtype([("lo", "<f4", 3), ("leftOrPrim", "<u4"), ("hi", "<f4", 3), ("packed", "<u4")])


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            from . import build_oracle
            build_oracle.build()
        lib = C.CDLL(str(LIB_PATH))
        vp, u32, i32, f32 = C.c_void_p, C.c_uint32, C.c_int, C.c_float
        sig = {
            "orc_create": (vp, []), "orc_destroy": (None, [vp]),
            "orc_add_mesh": (u32, [vp, vp]), "orc_add_instance": (u32, [vp, u32, vp, u32]),
            "orc_add_material": (u32, [vp, vp]), "orc_add_texture": (u32, [vp, vp]),
            "orc_remove_texture": (None, [vp, u32]), "orc_add_light": (u32, [vp, vp]),
            "orc_set_environment": (None, [vp, vp, f32, f32]), "orc_set_camera": (None, [vp, vp]),
            "orc_set_camera_ex": (None, [vp, vp]), "orc_set_settings": (None, [vp, vp]),
            "orc_commit": (u32, [vp]),
            "orc_render_f32": (i32, [vp, vp, u32, u32, u32, vp, i32]),
            "orc_render_f64": (i32, [vp, vp, u32, u32, u32, vp, i32]),
            "orc_render_f32_sum64": (i32, [vp, vp, u32, u32, u32, vp, i32]),
            "orc_trace": (i32, [vp, vp, u32, vp, i32]), "orc_trace_shadow": (i32, [vp, vp, u32, vp, i32]),
            "orc_trace_bruteforce": (i32, [vp, vp, u32, vp, vp, vp, i32]),
            "orc_bvh_build": (u32, [vp, u32, u32, vp, vp]), "orc_env_cdf": (f32, [vp, u32, u32, vp]),
            "orc_readback_f32": (None, [vp, u32, u32, vp]), "orc_resolve_rgba8": (None, [vp, u32, f32, u32, vp]),
            "orc_pcg4d": (None, [vp, u32, vp]), "orc_stats": (None, [vp, vp]),
            "orc_diff_of_products": (None, [vp, u32, vp]),
            "orc_mesh_attributes": (i32, [vp, u32, vp, u32, vp, vp, vp]),
            "orc_set_bruteforce": (None, [vp, i32]),
            "orc_set_all_leaf_instances": (None, [vp, i32]), "orc_unwalked_instances": (u32, [vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def diff_of_products(abcd):
    """float32 a*b - c*d by Kahan's FMA algorithm, as the watertight test's
    edge fallback computes it; abcd is (N, 4)."""
    x = np.ascontiguousarray(np.asarray(abcd, np.float32).reshape(-1, 4))
    out = np.empty(x.shape[0], np.float32)
    load().orc_diff_of_products(x.ctypes.data, x.shape[0], out.ctypes.data)
    return out


def _mesh_arrays(positions, indices, uvs):
    pos = np.ascontiguousarray(np.asarray(positions, np.float32).reshape(-1, 3))
    idx = np.ascontiguousarray(np.asarray(indices, np.uint32).reshape(-1))
    uv = None if uvs is None else np.ascontiguousarray(np.asarray(uvs, np.float32).reshape(-1, 2))
    return pos, idx, uv


def _attributes(fn, positions, indices, uvs):
    pos, idx, uv = _mesh_arrays(positions, indices, uvs)
    n = np.zeros((pos.shape[0], 4), np.float32)
    t = np.zeros((pos.shape[0], 4), np.float32)
    k = fn(_p(pos), pos.shape[0], _p(idx), idx.size, _p(uv), _p(n), _p(t))
    if k < 0:
        raise ValueError("mesh rejected")
    return n, (t if k else None)


def mesh_attributes(positions, indices, uvs=None):
    """The oracle's derived (normals, tangents or None) of a mesh given
    without normals, 4 floats per vertex each."""
    return _attributes(load().orc_mesh_attributes, positions, indices, uvs)


def load_ref_scene():
    """The reference's own scene store (compiled from its sources), or None."""
    global _ref_scene
    if _ref_scene is None and REF_SCENE_PATH.exists():
        lib = C.CDLL(str(REF_SCENE_PATH))
        lib.ref_mesh_attributes.restype = C.c_int
        lib.ref_mesh_attributes.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                            C.c_void_p]
        _ref_scene = lib
    return _ref_scene


def ref_mesh_attributes(positions, indices, uvs=None):
    """(normals, tangents or None) as the reference's Scene::addMesh derives
    them (Scene.cpp:13-92), from its compiled sources."""
    lib = load_ref_scene()
    if lib is None:
        raise RuntimeError("reference scene library not built (needs the reference checkout)")
    return _attributes(lib.ref_mesh_attributes, positions, indices, uvs)


def load_ref_envcdf():
    """The reference's own environment-CDF loop (compiled), or None."""
    global _ref_envcdf
    if _ref_envcdf is None and REF_ENVCDF_PATH.exists():
        lib = C.CDLL(str(REF_ENVCDF_PATH))
        lib.ref_env_cdf.restype = None
        lib.ref_env_cdf.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
        _ref_envcdf = lib
    return _ref_envcdf


def ref_env_cdf(rgba):
    """(cdf, integral) from the reference's Renderer.cpp:620-655 loop."""
    lib = load_ref_envcdf()
    if lib is None:
        raise RuntimeError("reference env-CDF library not built (needs the reference checkout)")
    px = np.ascontiguousarray(np.asarray(rgba, np.float32))
    h, w = px.shape[:2]
    cdf = np.empty(w * h + h, np.float32)
    integ = C.c_float()
    lib.ref_env_cdf(_p(px), w, h, _p(cdf), C.byref(integ))
    return cdf, integ.value


def load_ref_bvh():
    """The reference's own BvhBuilder (compiled from its sources), or None."""
    global _ref
    if _ref is None and REF_BVH_PATH.exists():
        lib = C.CDLL(str(REF_BVH_PATH))
        lib.ref_bvh_build.restype = C.c_uint32
        lib.ref_bvh_build.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
        _ref = lib
    return _ref


def bvh_build(aabbs, max_leaf, use_reference=False):
    """Binned-SAH BVH2 over (N, 6) AABBs: (nodes structured array, primOrder)."""
    a = np.ascontiguousarray(np.asarray(aabbs, np.float32).reshape(-1, 6))
    n = a.shape[0]
    nodes = np.zeros(max(2 * n, 1), NODE_DTYPE)
    order = np.zeros(max(n, 1), np.uint32)
    lib = load_ref_bvh() if use_reference else load()
    if lib is None:
        raise RuntimeError("reference BVH library not built (needs the reference checkout)")
    fn = lib.ref_bvh_build if use_reference else lib.orc_bvh_build
    count = fn(_p(a), n, max_leaf, _p(nodes), _p(order))
    return nodes[:count].copy(), order[:n].copy()


def env_cdf(rgba):
    px = np.ascontiguousarray(np.asarray(rgba, np.float32))
    h, w = px.shape[:2]
    cdf = np.empty(w * h + h, np.float32)
    integral = load().orc_env_cdf(_p(px), w, h, _p(cdf))
    return cdf, integral


def pcg4d(states):
    s = np.ascontiguousarray(np.asarray(states, np.uint32).reshape(-1, 4))
    out = np.empty_like(s)
    load().orc_pcg4d(_p(s), s.shape[0], _p(out))
    return out


def readback_f32(accum, frame_index):
    a = np.ascontiguousarray(np.asarray(accum, np.float32))
    out = np.empty_like(a)
    load().orc_readback_f32(_p(a), a.size // 4, frame_index, _p(out))
    return out


def resolve_rgba8(accum, exposure_ev=0.0, tonemap=abi.MRT_TONEMAP_ACES):
    a = np.ascontiguousarray(np.asarray(accum, np.float32))
    out = np.empty(a.shape, np.uint8)
    load().orc_resolve_rgba8(_p(a), a.size // 4, exposure_ev, tonemap, _p(out))
    return out


class OracleScene:
    """CPU oracle scene: same scene-building calls as miniraytrace_b200.Engine."""

    def __init__(self, width=1280, height=720):
        self.lib = load()
        self.h = self.lib.orc_create()
        self.width, self.height = width, height
        self._settings = dict(width=width, height=height, max_bounces=8, spp_limit=1024, exposure_ev=0.0,
                              firefly_clamp=50.0, tonemap=abi.MRT_TONEMAP_ACES)
        self._push_settings()

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _push_settings(self):
        s = self._settings
        d = abi.RenderSettings(width=s["width"], height=s["height"], maxBounces=s["max_bounces"],
                               sppLimit=s["spp_limit"], exposureEV=s["exposure_ev"],
                               fireflyClamp=s["firefly_clamp"], tonemap=s["tonemap"], denoise=0)
        self.lib.orc_set_settings(self.h, C.byref(d))

    def add_mesh(self, positions, indices, normals=None, uvs=None):
        d, keep = mesh_desc(positions, indices, normals, uvs)
        return self.lib.orc_add_mesh(self.h, C.byref(d))

    def add_instance(self, mesh_id, xform=None, material=0):
        xf = xform_rows(xform)
        return self.lib.orc_add_instance(self.h, mesh_id, _p(xf), material)

    def add_material(self, desc=None, **kw):
        d = desc if desc is not None else material_desc(**kw)
        return self.lib.orc_add_material(self.h, C.byref(d))

    def add_texture(self, pixels, fmt=abi.MRT_TEX_RGBA8_SRGB, generate_mips=False):
        d, keep = texture_desc(pixels, fmt, generate_mips)
        return self.lib.orc_add_texture(self.h, C.byref(d))

    def remove_texture(self, tex_id):
        self.lib.orc_remove_texture(self.h, tex_id)

    def add_light(self, desc=None, **kw):
        d = desc if desc is not None else light_desc(**kw)
        return self.lib.orc_add_light(self.h, C.byref(d))

    def set_environment(self, pixels, rotation=0.0, intensity=1.0):
        if pixels is None:
            self.lib.orc_set_environment(self.h, None, 0.0, 0.0)
            return
        d, keep = texture_desc(pixels, abi.MRT_TEX_RGBA32F)
        self.lib.orc_set_environment(self.h, C.byref(d), float(rotation), float(intensity))

    def set_camera(self, position=(0, 0, 5), target=(0, 0, 0), up=(0, 1, 0), fov_y_deg=45.0):
        d = abi.CameraDesc(position=abi.F3(*position), target=abi.F3(*target), up=abi.F3(*up),
                           fovYDeg=fov_y_deg)
        self.lib.orc_set_camera(self.h, C.byref(d))

    def set_camera_ex(self, projection=abi.MRT_CAMERA_PERSPECTIVE, position=(0, 0, 5), forward=(0, 0, -1),
                      up=(0, 1, 0), left=-1.0, right=1.0, bottom=-1.0, top=1.0):
        d = abi.CameraDescEx(projection=projection, position=abi.F3(*position), forward=abi.F3(*forward),
                             up=abi.F3(*up), left=left, right=right, bottom=bottom, top=top)
        self.lib.orc_set_camera_ex(self.h, C.byref(d))

    def set_render_settings(self, width=1280, height=720, max_bounces=8, spp_limit=1024, exposure_ev=0.0,
                            firefly_clamp=50.0, tonemap=abi.MRT_TONEMAP_ACES, denoise=True):
        self._settings = dict(width=width, height=height, max_bounces=max_bounces, spp_limit=spp_limit,
                              exposure_ev=exposure_ev, firefly_clamp=firefly_clamp, tonemap=tonemap)
        self.width, self.height = width, height
        self._push_settings()

    def commit(self):
        return self.lib.orc_commit(self.h)

    def set_bruteforce(self, mode: int):
        """Diagnostic: closest and shadow hits of the render calls
        (render_f32, render_f64, render_f32_sum64) by testing every triangle
        of every instance (1 = reference Moeller-Trumbore test, 2 = watertight
        test with the hit reported by the reference formula, 0 = BVH walk).
        trace_rays and trace_shadow_rays always walk the BVH."""
        self.lib.orc_set_bruteforce(self.h, int(mode))

    def set_all_leaf_instances(self, on: bool):
        """True: a TLAS leaf enters every instance it holds. False (default,
        the reference): only its first (intersect.glsl:116-121, 150-152), so
        the second instance of a 2-instance TLAS leaf, which Bvh.cpp:104 makes
        when SAH prefers it, is never traced."""
        self.lib.orc_set_all_leaf_instances(self.h, 1 if on else 0)

    def unwalked_instances(self) -> int:
        """After commit(): instances the reference traversal never enters."""
        return int(self.lib.orc_unwalked_instances(self.h))

    def render_f32(self, frame0, nframes, pixels=None, threads=8, accum=None):
        """Reference-order FP32 accumulation; returns (npix, 4) float32."""
        pix = None if pixels is None else np.ascontiguousarray(np.asarray(pixels, np.uint32))
        n = self.width * self.height if pix is None else pix.size
        a = accum if accum is not None else np.zeros((n, 4), np.float32)
        rc = self.lib.orc_render_f32(self.h, _p(pix), 0 if pix is None else pix.size, frame0, nframes, _p(a),
                                     threads)
        if rc:
            raise RuntimeError("oracle not committed")
        return a

    def render_f32_sum64(self, frame0, nframes, pixels=None, threads=8, sums=None):
        """FP32 paths summed in double in sample order (the GPU's accumulation);
        returns (npix, 3) float64 sums."""
        pix = None if pixels is None else np.ascontiguousarray(np.asarray(pixels, np.uint32))
        n = self.width * self.height if pix is None else pix.size
        s = sums if sums is not None else np.zeros((n, 3), np.float64)
        rc = self.lib.orc_render_f32_sum64(self.h, _p(pix), 0 if pix is None else pix.size, frame0, nframes, _p(s),
                                           threads)
        if rc:
            raise RuntimeError("oracle not committed")
        return s

    def render_f64(self, frame0, nframes, pixels=None, threads=8, sums=None):
        """FP64 evaluation of the same streams; returns (npix, 3) float64 sums."""
        pix = None if pixels is None else np.ascontiguousarray(np.asarray(pixels, np.uint32))
        n = self.width * self.height if pix is None else pix.size
        s = sums if sums is not None else np.zeros((n, 3), np.float64)
        rc = self.lib.orc_render_f64(self.h, _p(pix), 0 if pix is None else pix.size, frame0, nframes, _p(s),
                                     threads)
        if rc:
            raise RuntimeError("oracle not committed")
        return s

    def trace_rays(self, origins, dirs, t_max=1e30, threads=8):
        from miniraytrace_b200 import make_rays
        rays = make_rays(origins, dirs, t_max)
        hits = np.zeros(rays.shape[0], dtype=abi.HIT_DTYPE)
        self.lib.orc_trace(self.h, _p(rays), rays.shape[0], _p(hits), threads)
        return hits

    def trace_shadow_rays(self, origins, dirs, t_max=1e30, threads=8):
        from miniraytrace_b200 import make_rays
        rays = make_rays(origins, dirs, t_max)
        occ = np.zeros(rays.shape[0], np.uint32)
        self.lib.orc_trace_shadow(self.h, _p(rays), rays.shape[0], _p(occ), threads)
        return occ

    def trace_bruteforce(self, origins, dirs, t_max=1e30, threads=8):
        """(hits, second-nearest t, min barycentric) by brute force."""
        from miniraytrace_b200 import make_rays
        rays = make_rays(origins, dirs, t_max)
        n = rays.shape[0]
        hits = np.zeros(n, dtype=abi.HIT_DTYPE)
        t2 = np.zeros(n, np.float32)
        mb = np.zeros(n, np.float32)
        self.lib.orc_trace_bruteforce(self.h, _p(rays), n, _p(hits), _p(t2), _p(mb), threads)
        return hits, t2, mb

    def stats(self):
        out = np.zeros(5, np.uint32)
        self.lib.orc_stats(self.h, _p(out))
        return dict(nodes=int(out[0]), triangles=int(out[1]), instances=int(out[2]), tlasRoot=int(out[3]),
                    maxBlasDepth=int(out[4]))
