"""Rendering with the radiance cache (config 4's room at reduced sizes).
Switching the cache on or off starts a new accumulation; with it off the
path tracer is the plain one, bit for bit. With it on, the image is finite
and opaque, its mean stays within 15 % of a converged plain image (the cache
is biased, and its bias drifts as it trains), and at equal sample counts
after a short training warm-up its
relMSE against that image is well below the plain tracer's."""
import numpy as np
import pytest

from miniraytrace_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def rel_mse(x, r):
    return float(np.mean(np.sum((x - r) ** 2 / (r * r + 1e-2), -1)))


def test_cache_toggle_keeps_the_plain_path(gpu):
    w, h = 96, 64
    s = scenes.room(w, h)
    a = gpu.Engine(w, h)
    s.apply(a)
    a.render_frames(8)
    plain, n = a.read_accumulation()
    b = gpu.Engine(w, h)
    s.apply(b)
    b.set_radiance_cache(enabled=True)
    b.render_frames(8)
    img = b.read_framebuffer(abi.MRT_PIXEL_RGBA32F_LINEAR)
    assert np.isfinite(img).all() and (img[..., 3] == 1.0).all()
    assert b.read_accumulation()[1] == 8
    b.set_radiance_cache(enabled=False)  # a new accumulation, plain estimator
    assert b.read_accumulation()[1] == 0
    b.render_frames(8)
    again, m = b.read_accumulation()
    assert n == m == 8 and np.array_equal(plain, again)
    a.close()
    b.close()


def test_cached_render_beats_plain_at_equal_samples(gpu):
    # 320x180: about 1,800 training paths a sample. The cache is trained
    # online with a constant learning rate, and its overall brightness drifts
    # from one training round to the next (the gradient sums also use float
    # atomics, so no two runs are alike). Mean of the cached image over the
    # converged one, measured on a B200 (two seeds each): 64 warm-up samples
    # 1.007 to 1.054; 256 samples 0.85 to 0.95; 1,024 samples 0.95 to 1.03;
    # more training paths, a learning rate of 3e-3 or one training vertex
    # stayed within 0.88 to 1.01. The bound on the mean (15 %) therefore only
    # catches a gross error; the quality check is the relMSE, which stayed
    # within 0.42 to 0.49 of the plain tracer's in every one of those runs.
    w, h, spp = 320, 180, 64
    s = scenes.room(w, h)
    ref = gpu.Engine(w, h)
    s.apply(ref)
    ref.set_sample_stream(1 << 24, 1)
    ref.render_frames(4096)
    R = ref.read_framebuffer()[..., :3].astype(np.float64)
    ref.close()
    plain = gpu.Engine(w, h)
    s.apply(plain)
    plain.render_frames(spp)
    err_plain = rel_mse(plain.read_framebuffer()[..., :3].astype(np.float64), R)
    plain.close()
    e = gpu.Engine(w, h)
    s.apply(e)
    e.set_radiance_cache(enabled=True)
    e.render_frames(64)        # training warm-up
    e.set_sample_stream(0, 1)  # new accumulation, same trained cache
    e.render_frames(spp)
    X = e.read_framebuffer()[..., :3].astype(np.float64)
    e.close()
    err_cached = rel_mse(X, R)
    print(f"cached/converged mean {X.mean() / R.mean():.4f}, relMSE cached {err_cached:.3e} plain {err_plain:.3e}")
    assert np.isfinite(X).all()
    assert abs(X.mean() / R.mean() - 1.0) < 0.15, (X.mean(), R.mean())
    assert err_cached < 0.7 * err_plain, (err_cached, err_plain)
