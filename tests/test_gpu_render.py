"""Rendering parity and ABI semantics on the GPU, through the C ABI.

Image parity gate: at config 1 (256x256, 16 spp, same pcg4d streams, firefly
clamp equal on both sides) at least 99.9% of pixels match the FP32 oracle
within 1e-3 relative (per channel, |gpu - ref| <= 1e-3 * |ref| + 1e-6).

The known-answer tests restate the reference's GPU tests
(tests/camera_tests.cpp, commit_tests.cpp, tiling_regression_tests.cpp,
readback_bench_tests.cpp, material_texture_tests.cpp, gpu_selection_tests.cpp).
"""
import os
import time

import numpy as np
import pytest

from miniraytrace_b200 import abi, scenes

pytestmark = pytest.mark.gpu
THREADS = max(1, min(32, os.cpu_count() or 1))


def parity_fraction(img, ref, rtol=1e-3, atol=1e-6, report=8):
    d = np.abs(img[..., :3].astype(np.float64) - ref[..., :3].astype(np.float64))
    ok = (d <= rtol * np.abs(ref[..., :3]) + atol).all(-1)
    bad = np.argwhere(~ok)
    if len(bad) and report:
        rel = (d / (np.abs(ref[..., :3]) + atol)).max(-1)
        order = np.argsort(-rel[~ok])[:report]
        for y, x in bad[order]:
            print(f"  mismatch at ({x},{y}): gpu={img[y, x, :3]} ref={ref[y, x, :3]} rel={rel[y, x]:.3g}")
    return ok.mean()


def render_both(gpu, oracle_lib, s, spp):
    e = gpu.Engine(s.settings["width"], s.settings["height"])
    s.apply(e)
    for _ in range(spp):
        e.render_frame()
    img = e.read_framebuffer(abi.MRT_PIXEL_RGBA32F_LINEAR)
    o = oracle_lib.OracleScene(s.settings["width"], s.settings["height"])
    s.apply(o)
    o.commit()
    acc = o.render_f32(0, spp, threads=THREADS)
    ref = oracle_lib.readback_f32(acc, spp).reshape(img.shape)
    return e, img, ref, acc


def test_config1_image_parity(gpu, oracle_lib):
    s = scenes.box_sphere()
    e, img, ref, acc = render_both(gpu, oracle_lib, s, 16)
    assert (img[..., 3] == 1.0).all()
    assert np.isfinite(img).all()
    frac = parity_fraction(img, ref)
    print(f"config-1 parity: {frac * 100:.4f}% of pixels within 1e-3")
    assert frac >= 0.999
    # RGBA8: resolve of the same accumulation within 1 LSB
    rgba8 = e.read_framebuffer(abi.MRT_PIXEL_RGBA8_SRGB)
    ref8 = oracle_lib.resolve_rgba8(acc.reshape(img.shape), 0.0, abi.MRT_TONEMAP_LINEAR)
    close = (np.abs(rgba8.astype(int) - ref8.astype(int)) <= 1).all(-1).mean()
    assert close >= 0.999 and (rgba8[..., 3] == 255).all()
    e.close()


def bitexact_fraction(e, o, spp):
    """Fraction of pixels whose GPU FP64 accumulation equals, bit for bit, the
    oracle's double-precision sum of its FP32 paths (same sample streams)."""
    acc, n = e.read_accumulation()
    assert n == spp
    ref = o.render_f32_sum64(0, spp, threads=THREADS).reshape(acc.shape[0], acc.shape[1], 3)
    same = (acc[..., :3] == ref).all(-1)
    return same.mean()


def test_config1_paths_bitexact(gpu, oracle_lib):
    """Every GPU path of config 1 performs the oracle's FP32 arithmetic: the
    accumulated sums are identical bits, not merely within tolerance."""
    s = scenes.box_sphere(128, 128)
    e = gpu.Engine(128, 128)
    s.apply(e)
    e.render_frames(4)
    o = oracle_lib.OracleScene(128, 128)
    s.apply(o)
    o.commit()
    frac = bitexact_fraction(e, o, 4)
    print(f"config-1 bit-exact pixels: {frac * 100:.4f}%")
    assert frac >= 0.999
    e.close()


def test_environment_scene_parity(gpu, oracle_lib):
    """Config-2 features at a small size: env importance sampling + MIS,
    GGX conductors, dielectrics, instancing, diffuse terrain.

    Against the oracle's faithful restatement of the reference's BVH walk a
    few pixels differ. The reference's TLAS build (Bvh.cpp:104, leaf size 1)
    makes a 2-instance leaf when SAH prefers one, and its traversal
    (intersect.glsl:116-121, 150-152) enters only the first instance of a
    leaf, so one of this scene's 25 instances is never traced there. The
    engine's TLAS has one instance per leaf and traces every instance. With
    the oracle entering every instance of a leaf, or finding its closest and
    shadow hits by brute force (the watertight decision the kernel makes),
    every GPU path is bit-identical."""
    s = scenes.terrain(width=96, height=64, spp=4, grid=48, spheres=24, sky=(256, 128))
    e, img, ref, _ = render_both(gpu, oracle_lib, s, 4)
    frac = parity_fraction(img, ref)
    print(f"terrain parity vs reference BVH walk: {frac * 100:.4f}% of pixels within 1e-3")
    assert frac >= 0.995
    o = oracle_lib.OracleScene(96, 64)
    s.apply(o)
    o.commit()
    assert o.unwalked_instances() == 1
    o.set_all_leaf_instances(True)
    exact = bitexact_fraction(e, o, 4)
    print(f"terrain bit-exact pixels vs the walk entering every leaf instance: {exact * 100:.4f}%")
    assert exact >= 0.999
    o.set_all_leaf_instances(False)
    o.set_bruteforce(2)
    exact = bitexact_fraction(e, o, 4)
    print(f"terrain bit-exact pixels vs brute-force hits: {exact * 100:.4f}%")
    assert exact >= 0.999
    e.close()


def test_render_frames_equals_repeated_render_frame(gpu):
    s = scenes.box_sphere(64, 64)
    a = gpu.Engine(64, 64)
    s.apply(a)
    for _ in range(5):
        a.render_frame()
    b = gpu.Engine(64, 64)
    s.apply(b)
    info = b.render_frames(5)
    assert info["spp"] == 5
    ia, ib = a.read_framebuffer(), b.read_framebuffer()
    np.testing.assert_allclose(ia, ib, rtol=1e-6, atol=1e-7)
    acc, spp = b.read_accumulation()
    assert spp == 5 and (acc[..., 3] == 5).all()
    a.close()
    b.close()


def test_spp_limit_and_reset(gpu):
    s = scenes.box_sphere(32, 32)
    e = gpu.Engine(32, 32)
    s.apply(e)
    st = dict(s.settings)
    st["spp_limit"] = 3
    e.set_render_settings(**st)
    infos = [e.render_frame() for _ in range(5)]
    assert [i["spp"] for i in infos] == [1, 2, 3, 3, 3]
    assert [i["converged"] for i in infos] == [False, False, True, True, True]
    e.reset_accumulation()
    z = e.read_framebuffer()
    assert (z[..., :3] == 0).all() and (z[..., 3] == 1).all()
    assert e.render_frame()["spp"] == 1
    e.close()


# ---- reference tests/camera_tests.cpp ----------------------------------------------

def emissive_quad_engine(gpu, w, h, z):
    e = gpu.Engine(w, h)
    e.set_render_settings(width=w, height=h, max_bounces=0, spp_limit=1, denoise=False)
    s = 1000.0
    pos = np.array([[-s, -s, z], [s, -s, z], [s, s, z], [-s, -s, z], [s, s, z], [-s, s, z]], np.float32)
    mesh = e.add_mesh(pos, np.arange(6, dtype=np.uint32))
    mat = e.add_material(base_color=(0, 0, 0), emission=(1.0, 0.5, 0.25))
    e.add_instance(mesh, None, mat)
    return e


def render32(e):
    e.render_frame()
    return e.read_framebuffer(abi.MRT_PIXEL_RGBA32F_LINEAR)


def test_camera_ex_matches_legacy(gpu):
    legacy = emissive_quad_engine(gpu, 48, 48, -20.0)
    legacy.set_camera(position=(0, 0, 0), target=(0, 0, -1), up=(0, 1, 0), fov_y_deg=90.0)
    a = render32(legacy)
    ex = emissive_quad_engine(gpu, 48, 48, -20.0)
    ex.set_camera_ex(position=(0, 0, 0), forward=(0, 0, -1), up=(0, 1, 0), left=-1, right=1, bottom=-1, top=1)
    b = render32(ex)
    assert np.array_equal(a, b)
    assert np.array_equal(a[..., :3], np.broadcast_to(np.array([1.0, 0.5, 0.25], np.float32), a[..., :3].shape))


def test_orthographic_distance_invariance(gpu):
    imgs = []
    for eye in (0.0, 30.0):
        e = emissive_quad_engine(gpu, 32, 32, -50.0)
        e.set_camera_ex(projection=abi.MRT_CAMERA_ORTHOGRAPHIC, position=(0, 0, eye), forward=(0, 0, -1),
                        up=(0, 1, 0), left=-1, right=1, bottom=-1, top=1)
        imgs.append(render32(e))
    assert np.array_equal(imgs[0], imgs[1])


def test_asymmetric_crop(gpu):
    big = emissive_quad_engine(gpu, 64, 32, -20.0)
    big.set_camera_ex(forward=(0, 0, -1), up=(0, 1, 0), left=-1, right=1, bottom=-1, top=1)
    a = render32(big)
    crop = emissive_quad_engine(gpu, 32, 32, -20.0)
    crop.set_camera_ex(forward=(0, 0, -1), up=(0, 1, 0), left=0, right=1, bottom=-1, top=1)
    b = render32(crop)
    assert np.array_equal(a[:, 32:, :3], b[..., :3])


# ---- reference tests/commit_tests.cpp -------------------------------------------------

def small_engine(gpu, w=64, h=64, spp_limit=4):
    e = gpu.Engine(w, h)
    e.set_render_settings(width=w, height=h, spp_limit=spp_limit, denoise=False)
    return e


TRI = np.array([[-0.5, -0.5, 0.0], [0.5, -0.5, 0.0], [0.0, 0.5, 0.0]], np.float32)


def add_triangle(e, mat=0):
    mesh = e.add_mesh(TRI, np.arange(3, dtype=np.uint32))
    e.add_instance(mesh, None, mat)


def test_commit_noop(gpu):
    e = small_engine(gpu)
    st = e.commit()
    assert st["blasRebuilt"] == 0 and st["tlasRebuilt"] is False


def test_commit_rebuilds_once(gpu):
    e = small_engine(gpu)
    add_triangle(e)
    st = e.commit()
    assert st["blasRebuilt"] == 1 and st["tlasRebuilt"] is True
    st2 = e.commit()
    assert st2["blasRebuilt"] == 0 and st2["tlasRebuilt"] is False


def test_camera_only_commit_is_lightweight(gpu):
    e = small_engine(gpu)
    add_triangle(e)
    e.commit()
    e.set_camera(position=(0, 0, 6))
    st = e.commit()
    assert st["blasRebuilt"] == 0 and st["tlasRebuilt"] is False


def test_explicit_commit_matches_implicit(gpu):
    a = small_engine(gpu)
    add_triangle(a)
    a.commit()
    ia = a.render_frame()
    b = small_engine(gpu)
    add_triangle(b)
    ib = b.render_frame()
    assert ia["spp"] == ib["spp"]
    assert np.array_equal(a.read_framebuffer(), b.read_framebuffer())


# ---- reference tests/tiling_regression_tests.cpp ---------------------------------------

def test_small_emissive_triangle_visible(gpu):
    e = small_engine(gpu)
    pos = np.array([[-0.6, -0.6, 0.0], [0.6, -0.6, 0.0], [0.0, 0.6, 0.0]], np.float32)
    mesh = e.add_mesh(pos, np.arange(3, dtype=np.uint32))
    mat = e.add_material(base_color=(1.0, 0.2, 0.1), emission=(2.0, 0.4, 0.2))
    e.add_instance(mesh, None, mat)
    e.set_camera(position=(0, 0, 3), target=(0, 0, 0), up=(0, 1, 0), fov_y_deg=45.0)
    e.commit()
    for _ in range(4):
        e.render_frame()
    rgba8 = e.read_framebuffer(abi.MRT_PIXEL_RGBA8_SRGB)
    assert int(rgba8[..., 0].max()) > 10


# ---- reference tests/readback_bench_tests.cpp ---------------------------------------

def test_readback_1080p_fast_and_opaque(gpu):
    e = gpu.Engine(1920, 1080)
    e.set_render_settings(width=1920, height=1080, spp_limit=1, denoise=False)
    e.render_frame()
    buf = np.empty((1080, 1920, 4), np.float32)
    e.read_framebuffer(out=buf)
    t0 = time.perf_counter()
    for _ in range(20):
        e.read_framebuffer(out=buf)
    ms = (time.perf_counter() - t0) / 20 * 1e3
    print(f"1080p RGBA32F readback: {ms:.3f} ms/call")
    assert ms < 20.0
    assert (buf[..., 3] == 1.0).all()


def test_readback_rejects_small_dst(gpu):
    import ctypes as C
    e = gpu.Engine(16, 16)
    small = np.empty(16 * 16 * 4 - 1, np.float32)
    lib = gpu.load_library()
    r = lib.mrtReadFramebuffer(e.h, abi.MRT_PIXEL_RGBA32F_LINEAR, small.ctypes.data_as(C.c_void_p), small.nbytes)
    assert r == abi.MRT_ERROR_INVALID_ARGUMENT
    r = lib.mrtReadFramebuffer(e.h, abi.MRT_PIXEL_RGBA8_SRGB, small.ctypes.data_as(C.c_void_p), 16 * 16 * 4 - 1)
    assert r == abi.MRT_ERROR_INVALID_ARGUMENT


# ---- reference tests/material_texture_tests.cpp ---------------------------------------

def one_pixel(r, g, b):
    return np.array([[[r, g, b, 255]]], np.uint8)


def test_removed_material_falls_back(gpu):
    e = small_engine(gpu, 32, 32, 2)
    mat = e.add_material(base_color=(1, 0, 0))
    add_triangle(e, mat)
    e.commit()
    e.remove_material(mat)
    e.render_frame()


def test_texture_slot_recycling_and_fallback(gpu):
    e = small_engine(gpu, 32, 32, 2)
    t1 = e.add_texture(one_pixel(255, 0, 0), abi.MRT_TEX_RGBA8_UNORM)
    assert t1 != 0
    e.remove_texture(t1)
    t2 = e.add_texture(one_pixel(0, 255, 0), abi.MRT_TEX_RGBA8_UNORM)
    mat = e.add_material(base_color_tex=t2)
    add_triangle(e, mat)
    e.commit()
    e.render_frame()
    e.remove_texture(t2)
    e.commit()
    e.render_frame()


def test_texture_thrash_stays_bounded(gpu):
    e = small_engine(gpu, 32, 32, 2)
    prev = e.add_texture(one_pixel(10, 20, 30), abi.MRT_TEX_RGBA8_UNORM)
    e.commit()
    base = e.stats()["deviceBytes"]
    for i in range(300):
        e.remove_texture(prev)
        prev = e.add_texture(one_pixel(i % 256, 0, 0), abi.MRT_TEX_RGBA8_UNORM)
        assert prev != 0
        if i % 37 == 0:
            e.commit()
    e.commit()
    assert e.stats()["deviceBytes"] <= base + 4096
    e.render_frame()


def test_textured_material_parity(gpu, oracle_lib):
    """Base-color (sRGB), roughness (UNORM) and emission textures on the
    config-1 box, compared with the oracle."""
    s = scenes.box_sphere(64, 64)
    rng = np.random.default_rng(3)
    tex = rng.integers(0, 256, (8, 8, 4), dtype=np.uint8)
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    for m in s.meshes[:5]:
        m.uvs = uv
    e = gpu.Engine(64, 64)
    o = oracle_lib.OracleScene(64, 64)
    out = []
    for t in (e, o):
        s.apply(t)
        tid = t.add_texture(tex, abi.MRT_TEX_RGBA8_SRGB)
        tid2 = t.add_texture(tex, abi.MRT_TEX_RGBA8_UNORM)
        mid = t.add_material(base_color=(1, 1, 1), base_color_tex=tid, roughness_tex=tid2, emission=(0.2, 0.2, 0.2),
                             emission_tex=tid2)
        mesh = t.add_mesh(np.array([[-1, 0.01, 1], [1, 0.01, 1], [1, 0.01, -1], [-1, 0.01, -1]], np.float32),
                          np.array([0, 1, 2, 0, 2, 3], np.uint32), None, uv)
        t.add_instance(mesh, np.array([[0.5, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0.5, 0.4]], np.float32), mid)
        t.commit()
    for _ in range(4):
        e.render_frame()
    img = e.read_framebuffer()
    ref = oracle_lib.readback_f32(o.render_f32(0, 4, threads=THREADS), 4).reshape(img.shape)
    assert parity_fraction(img, ref) >= 0.999


def test_normal_map_parity(gpu, oracle_lib):
    """A normal-mapped material on uv-mapped meshes, compared with the oracle
    (which computes every mesh's tangents when it is stored, as the
    reference does). The engine computes tangents at commit for meshes drawn
    with a normal-mapped material: here its material gains the normal map
    after a first commit and the mesh is replaced under it afterwards; the
    oracle is given the final scene directly (same ids, same order)."""
    s = scenes.box_sphere(64, 64)
    rng = np.random.default_rng(5)
    nmap = np.empty((16, 16, 4), np.uint8)
    nmap[..., :2] = rng.integers(70, 186, (16, 16, 2))
    nmap[..., 2] = 220
    nmap[..., 3] = 255
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    for m in s.meshes[:5]:
        m.uvs = uv
    quad = np.array([[-1, 0.01, 1], [1, 0.01, 1], [1, 0.01, -1], [-1, 0.01, -1]], np.float32)
    tilted = quad + np.array([[0, 0.2, 0], [0, 0, 0], [0, 0.1, 0], [0, 0.3, 0]], np.float32)
    idx = np.array([0, 1, 2, 0, 2, 3], np.uint32)
    xf = np.array([[0.5, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0.5, 0.4]], np.float32)
    mat = dict(base_color=(0.9, 0.8, 0.7), roughness=0.4)

    e = gpu.Engine(64, 64)
    s.apply(e)
    tid = e.add_texture(nmap, abi.MRT_TEX_RGBA8_UNORM)
    mid = e.add_material(**mat)
    mesh = e.add_mesh(quad, idx, None, uv)
    e.add_instance(mesh, xf, mid)
    e.commit()
    e.render_frame()  # drawn without a normal map first
    e.update_material(mid, normal_tex=tid, **mat)
    e.commit()
    e.render_frame()
    e.update_mesh(mesh, tilted, idx, None, uv)
    e.commit()
    e.render_frames(4)
    img = e.read_framebuffer()

    o = oracle_lib.OracleScene(64, 64)
    s.apply(o)
    otid = o.add_texture(nmap, abi.MRT_TEX_RGBA8_UNORM)
    omid = o.add_material(normal_tex=otid, **mat)
    o.add_instance(o.add_mesh(tilted, idx, None, uv), xf, omid)
    o.commit()
    ref = oracle_lib.readback_f32(o.render_f32(0, 4, threads=THREADS), 4).reshape(img.shape)
    assert parity_fraction(img, ref) >= 0.999
    # the normal map changes the image (the comparison is not vacuous)
    e.update_material(mid, **mat)
    e.commit()
    e.render_frames(4)
    assert parity_fraction(e.read_framebuffer(), ref, report=0) < 0.999


def test_point_and_rect_lights_parity(gpu, oracle_lib):
    s = scenes.box_sphere(64, 64)
    s.lights = [dict(type=abi.MRT_LIGHT_POINT, position=(0.3, 1.6, 0.2), radiance=(5.0, 4.0, 3.0)),
                dict(type=abi.MRT_LIGHT_RECT, corner=(-0.4, 1.99, -0.4), edge0=(0.8, 0, 0), edge1=(0, 0, 0.8),
                     radiance=(6.0, 6.0, 6.0), two_sided=True)]
    e, img, ref, _ = render_both(gpu, oracle_lib, s, 4)
    assert parity_fraction(img, ref) >= 0.999


# ---- reference tests/gpu_selection_tests.cpp -------------------------------------------

def test_out_of_range_gpu_index_fails_clearly(gpu):
    with pytest.raises(gpu.MrtError) as e:
        gpu.Engine(16, 16, gpu_index1=10000)
    assert e.value.code == abi.MRT_ERROR_VULKAN_INIT
    assert "out of range" in gpu.last_error()


def test_env_cdf_kernel_matches_oracle(gpu, oracle_lib):
    e = gpu.Engine(16, 16)
    for w, h in ((64, 32), (2048, 1024), (4096, 2048)):
        sky = scenes.procedural_sky(w, h)
        cdf, integ = e.build_env_cdf(sky)
        rcdf, rinteg = oracle_lib.env_cdf(sky)
        # same sequential double sums as the reference: identical bits
        assert np.array_equal(cdf, rcdf), (w, h, int(np.sum(cdf != rcdf)))
        assert np.float32(integ) == np.float32(rinteg)
    e.close()


def test_queued_frames_match_immediate_rendering(gpu):
    """mrtRenderFrame queues samples and renders them as one wave (when a
    full wave is queued or something reads the results); every observable
    result equals rendering each frame at once: accumulation, frame info,
    reads between frames, and a camera change dropping queued samples."""
    s = scenes.box_sphere(64, 64)
    a = gpu.Engine(64, 64)
    s.apply(a)
    b = gpu.Engine(64, 64)
    s.apply(b)
    # 70 frames: one full 64-sample wave flushes by itself, 6 stay queued
    infos = [a.render_frame() for _ in range(70)]
    assert [i["spp"] for i in infos] == list(range(1, 71))
    b.render_frames(70)
    acc_a, spp_a = a.read_accumulation()
    acc_b, spp_b = b.read_accumulation()
    assert spp_a == spp_b == 70
    assert np.array_equal(acc_a, acc_b)
    # reads in between flush what is queued
    for _ in range(3):
        a.render_frame()
    b.render_frames(3)
    assert np.array_equal(a.read_framebuffer(), b.read_framebuffer())
    assert a.stats()["lastRenderSpp"] == 3
    # a camera change drops queued samples: the reset would erase them
    for _ in range(4):
        a.render_frame()
    cam = dict(s.camera)
    cam["position"] = tuple(np.asarray(cam["position"]) * 1.1)
    a.set_camera(**cam)
    b.set_camera(**cam)
    assert a.render_frame()["spp"] == 1
    b.render_frames(1)
    assert np.array_equal(a.read_accumulation()[0], b.read_accumulation()[0])
    a.close()
    b.close()


def test_incremental_geometry_commit_matches_fresh_engine(gpu):
    """Geometry commits keep every mesh on the device and re-assemble the
    scene arrays there: after one mesh changes (a heightfield large enough
    for the device BVH builder) and another is removed, the unchanged meshes'
    device copies are reused, and the image equals that of an engine given
    the final scene at once."""
    s = scenes.terrain(96, 64, spp=4, grid=300, spheres=24)
    pos2, idx2, nrm2, _ = scenes.heightfield(300, 0.15, seed=8)
    extra_p, extra_i, extra_n = scenes.icosphere(2)
    a = gpu.Engine(96, 64)
    ids = s.apply(a)
    extra = a.add_mesh(extra_p * 0.05 + np.float32([0.0, 0.3, 0.0]), extra_i, extra_n)
    a.add_instance(extra)
    a.render_frames(2)
    a.update_mesh(ids["meshes"][0], pos2, idx2, nrm2)
    a.remove_mesh(extra)
    st = a.commit()
    assert st["blasRebuilt"] == 1
    a.render_frames(4)
    b = gpu.Engine(96, 64)
    ids_b = s.apply(b)
    b.update_mesh(ids_b["meshes"][0], pos2, idx2, nrm2)
    b.render_frames(4)
    acc_a, spp_a = a.read_accumulation()
    acc_b, spp_b = b.read_accumulation()
    assert spp_a == spp_b == 4
    assert np.array_equal(acc_a, acc_b)
    # trace queries see the same triangles (ids in the mesh's own index order)
    rng = np.random.default_rng(3)
    o = np.tile(np.float32([0.0, 0.6, 0.0]), (512, 1))
    d = rng.normal(size=(512, 3)).astype(np.float32)
    d[:, 1] = -np.abs(d[:, 1])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    ha, hb = a.trace_rays(o, d), b.trace_rays(o, d)
    assert np.array_equal(ha["prim"], hb["prim"]) and np.array_equal(ha["t"], hb["t"])
    a.close()
    b.close()


def test_l2_bandwidth_probe(gpu):
    """mrtxMeasureL2Bandwidth returns a plausible L2 read bandwidth (above a
    tenth of the HBM copy rate, below 100 TB/s) and frees its buffer."""
    e = gpu.Engine(16, 16)
    base = e.stats()["deviceBytes"]
    g = e.measure_l2_bandwidth()
    assert 600.0 < g < 100000.0, g
    assert e.stats()["deviceBytes"] == base
    e.close()



def test_managed_smoke_and_engine_lifecycle_cycles(gpu):
    """The reference's managed smoke test (rhino/MiniRaytrace.Smoke/
    Program.cs:33-130) through the C ABI: an emissive triangle at 64x64 and
    4 spp (commit rebuilds exactly one BLAS, spp 4, a non-black RGBA8 image,
    RGBA32F alpha 1), then 30 engine lifecycles on worker threads as its
    render sessions run them (created on the render thread, a few frames of
    an empty scene read back, destroyed). Every cycle completes, and the
    device memory the process holds returns to its level after the first."""
    import threading

    import torch

    e = gpu.Engine(64, 64)
    m = e.add_mesh(np.array([[-0.6, -0.6, 0], [0.6, -0.6, 0], [0, 0.6, 0]], np.float32),
                   np.array([0, 1, 2], np.uint32))
    mat = e.add_material(base_color=(1.0, 0.2, 0.1), emission=(2.0, 0.4, 0.2))
    assert e.add_instance(m, None, mat) != 0
    e.set_camera(position=(0, 0, 3), target=(0, 0, 0))
    e.set_render_settings(width=64, height=64, spp_limit=4, denoise=False)
    assert e.commit()["blasRebuilt"] == 1
    info = None
    for _ in range(4):
        info = e.render_frame()
    assert info["spp"] == 4
    rgba8 = e.read_framebuffer(abi.MRT_PIXEL_RGBA8_SRGB)
    assert (rgba8[..., :3] > 10).any()
    assert (e.read_framebuffer(abi.MRT_PIXEL_RGBA32F_LINEAR)[..., 3] == 1.0).all()
    e.close()

    def cycle(out):
        try:
            s = gpu.Engine(48, 48)
            s.set_render_settings(width=48, height=48, denoise=False)
            for _ in range(3):
                s.commit()
                s.render_frame()
                img = s.read_framebuffer(abi.MRT_PIXEL_RGBA32F_LINEAR)
            s.close()
            out.append(bool(np.isfinite(img).all() and (img[..., 3] == 1.0).all()))
        except Exception as ex:  # reported below
            out.append(ex)

    free = []
    for i in range(30):
        out = []
        t = threading.Thread(target=cycle, args=(out,))
        t.start()
        t.join(timeout=60)
        assert not t.is_alive() and out == [True], (i, out)
        free.append(torch.cuda.mem_get_info()[0])
    assert free[0] - min(free[1:]) < 64 << 20, [f >> 20 for f in free]
