"""The opt-in denoiser (mrtxSetDenoiser), in place of the reference's optional
OIDN filter (core/src/post/Denoiser.cpp, scheduled by Renderer.cpp:845-884).

- Its guides are the reference's first-hit AOVs (pathtrace.comp:130-167):
  checked on a quad of known albedo and normal.
- The filter is checked against a numpy restatement of the same a-trous
  passes on the engine's own accumulation and guides (tolerance: the GPU
  uses the fast exp / pow intrinsics, so 1e-4 of the image's peak, and 1e-3
  relative for 99.9% of the values).
- It lowers the error against a converged image.
- It is off by default and follows the reference's display semantics: RGBA8
  reads show it from 8 samples on, frame infos report `denoised`, a reset
  clears it, and RGBA32F reads stay the raw mean."""
import numpy as np
import pytest

from miniraytrace_b200 import abi, scenes

pytestmark = pytest.mark.gpu

B3 = np.array([0.375, 0.25, 0.0625], np.float32)


def denoise_numpy(mean, albedo, normal_depth, samples, iterations=5, sigma_color=1.0, normal_power=64.0,
                  sigma_albedo=0.1, sigma_depth=0.1, floor=0.01):
    """The a-trous passes of csrc/cuda/denoise.cu in float32 numpy."""
    h, w = mean.shape[:2]
    al = albedo[..., :3].astype(np.float32)
    alf = np.maximum(al, np.float32(floor))
    irr = (mean[..., :3].astype(np.float32) / alf).astype(np.float32)
    n = normal_depth[..., :3].astype(np.float32)
    ln = np.sqrt((n * n).sum(-1, keepdims=True))
    un = np.where(ln > 0, n / np.where(ln > 0, ln, 1), 0).astype(np.float32)
    z = normal_depth[..., 3].astype(np.float32)
    hit = z > 0
    src = irr
    ys, xs = np.mgrid[0:h, 0:w]
    for i in range(iterations):
        step = 1 << i
        inv_c2 = np.float32(1.0 / (sigma_color * sigma_color / samples * 2.0 ** -i))
        cc = np.log1p(np.maximum(src * alf, 0.0)).astype(np.float32)
        inv_d = np.where(hit, 1.0 / (sigma_depth * np.where(hit, z, 1) * step), 0).astype(np.float32)
        acc = np.zeros_like(src)
        wsum = np.zeros((h, w), np.float32)
        for dy in range(-2, 3):
            for dx in range(-2, 3):
                yy, xx = ys + dy * step, xs + dx * step
                ok = (yy >= 0) & (yy < h) & (xx >= 0) & (xx < w)
                yq, xq = np.clip(yy, 0, h - 1), np.clip(xx, 0, w - 1)
                same = ok & (hit[yq, xq] == hit)
                wgt = B3[abs(dx)] * B3[abs(dy)] * np.exp(-((cc - cc[yq, xq]) ** 2).sum(-1) * inv_c2)
                nd = np.maximum((un * un[yq, xq]).sum(-1), 0.0)
                g = nd ** normal_power * np.exp(-((al - al[yq, xq]) ** 2).sum(-1) / sigma_albedo ** 2) * \
                    np.exp(-np.abs(z - z[yq, xq]) * inv_d)
                wgt = np.where(same, np.where(hit, wgt * g, wgt), 0).astype(np.float32)
                acc += wgt[..., None] * src[yq, xq]
                wsum += wgt
        src = (acc / wsum[..., None]).astype(np.float32)
    return src * alf


def rel_mse(x, ref):
    return float(np.mean((x[..., :3] - ref[..., :3]) ** 2 / (ref[..., :3] ** 2 + 1e-2)))


def make_engine(gpu, scene, stream=0):
    e = gpu.Engine(scene.settings["width"], scene.settings["height"])
    scene.apply(e)
    if stream:
        e.set_sample_stream(stream, 1)
    e.commit()
    return e


def test_guides_of_a_facing_quad(gpu):
    s = scenes.SceneSpec("quad")
    pos, idx = scenes.quad((-4, -4, 0), (4, -4, 0), (4, 4, 0), (-4, 4, 0))
    s.meshes.append(scenes.MeshSpec(pos, idx))
    s.materials.append(dict(base_color=(0.3, 0.5, 0.7), roughness=1.0, metallic=0.0))
    s.instances.append((0, None, 0))
    s.lights.append(dict(type=abi.MRT_LIGHT_SUN, direction=(0.0, 0.0, -1.0), radiance=(1.0, 1.0, 1.0)))
    s.camera = dict(position=(0.0, 0.0, 2.0), target=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), fov_y_deg=40.0)
    s.settings = dict(width=64, height=48, max_bounces=4)
    e = make_engine(gpu, s)
    e.set_denoiser(enabled=True)
    albedo, nd = e.read_denoiser_guides()
    assert np.allclose(albedo[..., :3], [0.3, 0.5, 0.7], atol=1e-6)
    assert np.all(albedo[..., 3] == 1.0)
    assert np.allclose(nd[..., :3], [0.0, 0.0, 1.0], atol=1e-6)  # faces the camera
    # distance to the plane z = 0 along the pixel's rays: 2 at the centre,
    # up to 2 / cos(half the diagonal field of view) at the corners
    assert abs(nd[24, 32, 3] - 2.0) < 0.01
    t = np.tan(np.radians(20.0))
    corner = 2.0 * np.sqrt(1.0 + t * t + (t * 64 / 48) ** 2)
    assert np.all(nd[..., 3] >= 2.0 - 1e-4) and np.all(nd[..., 3] <= corner + 1e-3)
    e.close()


def test_filter_matches_numpy_restatement(gpu):
    s = scenes.box_sphere(96, 80, max_bounces=6)
    e = make_engine(gpu, s)
    e.set_denoiser(enabled=True)
    e.render_frames(16)
    acc, n = e.read_accumulation()
    assert n == 16
    mean = acc[..., :3] / acc[..., 3:4]
    albedo, nd = e.read_denoiser_guides()
    got = e.read_denoised()
    want = denoise_numpy(mean, albedo, nd, 16)
    assert np.all(got[..., 3] == 1.0)
    peak = float(np.abs(want).max())
    err = np.abs(got[..., :3] - want)
    assert float(err.max()) <= 1e-4 * peak, float(err.max() / peak)
    assert np.mean(err <= 1e-3 * np.abs(want) + 1e-6 * peak) >= 0.999
    e.close()


def test_denoiser_lowers_error_against_converged_image(gpu):
    # firefly clamp 10 in both renders: unclamped, the sun's caustics off the
    # metal sphere leave isolated outliers that no edge-avoiding filter
    # removes and that dominate the relMSE
    s = scenes.box_sphere(128, 128, max_bounces=6, firefly_clamp=10.0)
    ref_e = make_engine(gpu, s, stream=1 << 24)
    ref_e.set_render_settings(**dict(s.settings, spp_limit=4096))
    ref_e.render_frames(4096)
    ref = ref_e.read_framebuffer()
    ref_e.close()
    e = make_engine(gpu, s)
    e.set_denoiser(enabled=True)
    e.render_frames(16)
    noisy = e.read_framebuffer()
    den = e.read_denoised()
    err_noisy, err_den = rel_mse(noisy, ref), rel_mse(den, ref)
    assert err_den < 0.5 * err_noisy, (err_noisy, err_den)
    e.close()


def test_display_schedule_frame_info_and_defaults(gpu):
    s = scenes.box_sphere(64, 64, max_bounces=6)
    s.settings = dict(s.settings, denoise=True)
    raw = make_engine(gpu, s)
    e = make_engine(gpu, s)
    rgba8 = abi.MRT_PIXEL_RGBA8_SRGB
    e.set_denoiser(enabled=True)
    # before 8 samples the display read is the raw resolve
    for _ in range(4):
        assert not raw.render_frame()["denoised"]  # off by default
        assert not e.render_frame()["denoised"]
    assert np.array_equal(e.read_framebuffer(rgba8), raw.read_framebuffer(rgba8))
    for _ in range(4):
        raw.render_frame()
        e.render_frame()
    # 8 samples: the display read shows the denoised image ...
    assert not np.array_equal(e.read_framebuffer(rgba8), raw.read_framebuffer(rgba8))
    assert e.render_frame()["denoised"]
    assert not raw.render_frame()["denoised"]
    # ... while the linear read stays the raw mean
    assert np.array_equal(e.read_framebuffer(), raw.read_framebuffer())
    # the render setting `denoise` turns it off, as in the reference
    e.set_render_settings(**dict(s.settings, denoise=False))
    e.commit()
    assert not e.render_frame()["denoised"]
    # a reset clears it
    e.set_render_settings(**dict(s.settings, denoise=True))
    e.commit()
    e.reset_accumulation()
    assert not e.render_frame()["denoised"]
    with pytest.raises(Exception):
        e.set_denoiser(enabled=True, iterations=11)
    e.set_denoiser(enabled=False)
    with pytest.raises(Exception):
        e.read_denoised()
    raw.close()
    e.close()
