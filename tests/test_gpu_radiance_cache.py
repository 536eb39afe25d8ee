"""Radiance cache network on the GPU against the oracle's numpy restatement
of the same network (oracle/radiance_cache.py): hash-grid + spherical-harmonics encoding and 5 x 64 ReLU MLP
outputs, the direction of one Adam step (its first step moves every
parameter by +-learning rate, opposite to the gradient's sign), and that
training fits a smooth function. Inference runs on the tensor cores with
BF16 operands and FP32 sums: its outputs are compared with numpy rounding
the encoding, the weights and each hidden activation to BF16 (round to
nearest even) and summing in FP64: 99.9 % of the outputs within 5e-3
relative + 2e-4 absolute (FP32 sums in another order, device rsqrt), all
within 1e-2 relative + 2e-3 absolute (the odd hidden activation whose FP32
sum lands on the other side of a BF16 rounding boundary moves by one BF16
step), and all within 3e-2 of the output scale of the FP32 network.
Training runs on the tensor cores too (BF16 activations, weights and
back-propagated gradients, FP32 sums): one Adam step is compared by sign
with gradients from numpy doing the same roundings, where they are above
1e-3 of their layer's largest."""
import numpy as np
import pytest

from miniraytrace_b200 import abi
from oracle.radiance_cache import encode, forward, forward_bf16, gradients_bf16

pytestmark = pytest.mark.gpu

LR = 1e-2


def assert_bf16_close(out, ref, msg=""):
    near = np.isclose(out, ref, rtol=5e-3, atol=2e-4)
    assert near.mean() >= 0.999, (msg, near.size - near.sum())
    np.testing.assert_allclose(out, ref, rtol=1e-2, atol=2e-3, err_msg=msg)


def random_features(rng, n, lo, hi):
    F = np.zeros((n, 16), np.float32)
    F[:, :3] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    F[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    nn = rng.normal(size=(n, 3))
    F[:, 6:9] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    F[:, 9] = rng.uniform(0, 1, n)
    F[:, 10:13] = rng.uniform(0, 1, (n, 3))
    return F


def random_params(rng):
    grid = (rng.normal(size=abi.CACHE_GRID_FLOATS) * 0.5).astype(np.float32)
    mlp = (rng.uniform(-1, 1, abi.CACHE_MLP_FLOATS) * np.sqrt(6.0 / 128)).astype(np.float32)
    mlp.reshape(6, 64, 64)[5][3:] = 0
    return grid, mlp


LO = np.array([-2.0, 0.0, 1.0], np.float32)
HI = np.array([3.0, 4.0, 2.5], np.float32)


@pytest.fixture()
def engine(gpu):
    e = gpu.Engine(16, 16)
    e.set_radiance_cache(enabled=False, bounds=(LO, HI), learning_rate=LR)
    yield e
    e.close()


def test_query_matches_numpy(engine):
    rng = np.random.default_rng(1)
    grid, mlp = random_params(rng)
    engine.cache_params(grid, mlp)
    F = random_features(rng, 2000, LO, HI)
    out = engine.cache_query(F)
    enc, _ = encode(F, grid, LO, HI)
    ref = forward_bf16(enc, mlp)
    assert ref.max() > 0.1
    assert_bf16_close(out, ref)
    fp32 = np.maximum(forward(enc, mlp)[0], 0.0)
    assert np.abs(out - fp32).max() < 3e-2 * np.abs(fp32).max()


def test_query_tiles_and_ragged_counts(engine):
    """Counts around the 128-query tile and more tiles than resident CTAs:
    every query's output is its own (the same as a query alone)."""
    rng = np.random.default_rng(4)
    grid, mlp = random_params(rng)
    engine.cache_params(grid, mlp)
    F = random_features(rng, 148 * 3 * 128 * 2 + 77, LO, HI)
    ref = forward_bf16(encode(F, grid, LO, HI)[0], mlp)
    for n in (1, 127, 128, 129, 1000, F.shape[0]):
        out = engine.cache_query(F[:n])
        assert_bf16_close(out, ref[:n], str(n))


def test_one_adam_step_follows_numpy_gradients(engine):
    rng = np.random.default_rng(2)
    grid, mlp = random_params(rng)
    engine.cache_params(grid, mlp)
    F = random_features(rng, 256, LO, HI)
    targets = rng.uniform(0, 2, (256, 3)).astype(np.float32)
    engine.cache_train(F, targets, steps=1)
    grid1, mlp1 = engine.cache_params()
    gW, gG = gradients_bf16(F, targets.astype(np.float64), grid, mlp, LO, HI)
    for name, p0, p1, g in (("mlp", mlp, mlp1, gW), ("grid", grid, grid1, gG)):
        step = p1.astype(np.float64) - p0
        big = np.abs(g) > 1e-3 * np.abs(g).max()
        assert big.sum() > 100, name
        # Adam's first step: -lr * g / (|g| + eps)
        np.testing.assert_allclose(step[big], -LR * np.sign(g[big]), rtol=1e-3, atol=1e-6, err_msg=name)
        # untouched parameters stay put
        assert np.all(step[g == 0] == 0), name


def test_training_fits_a_smooth_function(engine):
    rng = np.random.default_rng(3)
    F = random_features(rng, 16384, LO, HI)
    x, z = F[:, 0], F[:, 2]
    targets = np.stack([0.5 + 0.4 * np.sin(2 * x) * np.cos(3 * z), 0.3 + 0.2 * F[:, 4], 0.2 + 0.1 * F[:, 10]], 1)
    first = engine.cache_train(F, targets, steps=1)
    for _ in range(20):
        last = engine.cache_train(F, targets, steps=20) / 20
    assert last < first / 20, (first, last)
    assert np.mean(np.abs(engine.cache_query(F) - targets)) < 0.03
    # points it was not trained on: the fine hash levels memorise the 16k
    # training points, the coarse levels and the network still generalise
    held = random_features(rng, 2000, LO, HI)
    pred = engine.cache_query(held)
    want = np.stack([0.5 + 0.4 * np.sin(2 * held[:, 0]) * np.cos(3 * held[:, 2]), 0.3 + 0.2 * held[:, 4],
                     0.2 + 0.1 * held[:, 10]], 1)
    assert np.mean(np.abs(pred - want)) < 0.1
