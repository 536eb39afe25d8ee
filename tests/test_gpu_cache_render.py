"""Rendering with the radiance cache (config 4's room at reduced sizes).
Switching the cache on or off starts a new accumulation; with it off the
path tracer is the plain one, bit for bit. With it on (default training
schedule: the learning rate halves every 96 Adam steps down to 3e-4, and
queries read a moving average of the weights), after a training warm-up
the image is finite and opaque, its mean stays within 3 % of a converged
plain image for two cache seeds, and its relMSE against that image is at
most half the plain tracer's at equal sample counts."""
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


@pytest.mark.parametrize("seed", [1, 2])
def test_cached_render_beats_plain_at_equal_samples(gpu, seed):
    # 320x180: about 1,800 training paths a sample, one Adam step a sample.
    # With a constant learning rate (1e-2) the cache's weights kept wandering
    # and the cached image's mean over the converged one ranged 0.85 to 1.20
    # between runs (four seeds, warm-ups of 64 and 256 samples); averaging
    # the weights alone did not change that. Decaying the rate settled it:
    # 0.995 to 1.003 with averaging once the rate reached 3e-4 (four seeds),
    # relMSE 0.30 to 0.32 of the plain tracer's (B200 measurements).
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
    e.set_radiance_cache(enabled=True, seed=seed)
    e.render_frames(512)       # training warm-up: the rate has decayed to its floor (3e-4)
    e.set_sample_stream(0, 1)  # new accumulation, same trained cache
    e.render_frames(spp)
    X = e.read_framebuffer()[..., :3].astype(np.float64)
    e.close()
    err_cached = rel_mse(X, R)
    print(f"seed {seed}: cached/converged mean {X.mean() / R.mean():.4f}, relMSE cached {err_cached:.3e} "
          f"plain {err_plain:.3e}")
    assert np.isfinite(X).all()
    assert abs(X.mean() / R.mean() - 1.0) < 0.03, (X.mean(), R.mean())
    assert err_cached < 0.5 * err_plain, (err_cached, err_plain)
