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
from oracle.radiance_cache import bf16, encode, forward, forward_bf16, gradients_bf16

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
    e.set_cache_averaging(0.0)  # queries read the live weights (averaging has its own test)
    e.set_cache_schedule(0.0, 0.0)  # a constant learning rate
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


def touched_grid_entries(F, grid):
    """Flat indices of the grid floats some sample's corners reach (both
    features of each corner entry), from the oracle's encoding."""
    _, corners = encode(F, grid, LO, HI)
    idx = np.unique(np.concatenate([i for lvl in corners for i, _ in lvl]))
    return np.concatenate([2 * idx, 2 * idx + 1])


@pytest.mark.parametrize("n", [1, 127, 129, 16384])
def test_gradients_match_oracle_value_by_value(engine, n):
    """The training kernels' raw gradients of one batch (before Adam) against
    the oracle's gradients with the same BF16 roundings.

    Tolerance: per MLP layer, 99.9% of the weights' gradients within 1e-2 of
    that layer's largest |gradient| (FP32 sums in another order move the odd
    activation or back-propagated value across a BF16 rounding boundary,
    one BF16 step = 2^-8 relative), all within 5e-2 of it; the output
    layer's unused rows exactly 0. Per hash-grid level, 99.9% of the
    entries the batch touches within 1e-2 of the level's largest, all
    within 0.25 of it (a level sums many samples per entry, and at 16,384
    samples the odd entry collects a sample whose activation rounded the
    other way: 0.13 was seen once); every entry no sample reaches exactly
    0. A wrong chain-rule factor or a mis-scaled scatter moves every entry,
    so the 99.9% bound catches it.
    The mean loss within 1e-2 relative (a single sample's output moves by
    a BF16 step when one of its activations rounds the other way)."""
    rng = np.random.default_rng(40 + n)
    grid, mlp = random_params(rng)
    engine.cache_params(grid, mlp)
    F = random_features(rng, n, LO, HI)
    targets = rng.uniform(0, 2, (n, 3)).astype(np.float32)
    g_grid, g_mlp, loss = engine.cache_gradients(F, targets)
    want_mlp, want_grid = gradients_bf16(F, targets.astype(np.float64), grid, mlp, LO, HI)

    got_w = g_mlp.reshape(6, 64, 64).astype(np.float64)
    want_w = want_mlp.reshape(6, 64, 64)
    assert np.all(got_w[5][3:] == 0)
    for layer in range(6):
        rows = 3 if layer == 5 else 64
        a, b = got_w[layer][:rows], want_w[layer][:rows]
        scale = np.abs(b).max()
        assert scale > 0, layer
        close = np.abs(a - b) <= 1e-2 * scale
        assert close.mean() >= 0.999, (n, layer, int((~close).sum()))
        assert np.abs(a - b).max() <= 5e-2 * scale, (n, layer, np.abs(a - b).max() / scale)

    touched = touched_grid_entries(F, grid)
    untouched = np.ones(g_grid.size, bool)
    untouched[touched] = False
    assert np.all(g_grid[untouched] == 0), int(np.count_nonzero(g_grid[untouched]))
    per_level = g_grid.size // 16
    for level in range(16):
        sel = touched[(touched >= level * per_level) & (touched < (level + 1) * per_level)]
        a, b = g_grid[sel].astype(np.float64), want_grid[sel]
        scale = np.abs(b).max()
        if scale == 0:
            assert np.all(a == 0), level
            continue
        close = np.abs(a - b) <= 1e-2 * scale
        assert close.mean() >= 0.999, (n, level, int((~close).sum()))
        assert np.abs(a - b).max() <= 0.25 * scale, (n, level, np.abs(a - b).max() / scale)

    enc, _ = encode(F, grid, LO, HI)
    W = mlp.reshape(6, 64, 64)
    h = bf16(enc)
    for layer in range(5):
        h = bf16(np.maximum(h @ bf16(W[layer]).T, 0.0))
    y = h @ bf16(W[5][:3]).T
    want_loss = np.mean((y - targets) ** 2 / (y * y + 0.01))
    assert abs(loss - want_loss) <= 1e-2 * want_loss, (loss, want_loss)

    # nothing moved: the parameters are as written
    grid1, mlp1 = engine.cache_params()
    assert np.array_equal(grid1, grid) and np.array_equal(mlp1, mlp)


def test_weight_average_follows_its_formula(engine):
    """Averaging on: one Adam step moves the live weights; the average takes
    them with weight 1 - d, d = min(decay, (1 + k) / (10 + k)) = 2/11 at the
    first step (k = 1), entries the batch did not touch keep their value, and
    queries read the average. Tolerance: queries as in
    test_query_matches_numpy (the average itself is one FP32 blend)."""
    rng = np.random.default_rng(6)
    grid, mlp = random_params(rng)
    engine.set_cache_averaging(0.9)
    engine.cache_params(grid, mlp)  # restarts the average at these weights
    F = random_features(rng, 512, LO, HI)
    targets = rng.uniform(0, 2, (512, 3)).astype(np.float32)
    engine.cache_train(F, targets, steps=1)
    grid1, mlp1 = engine.cache_params()
    d = np.float32(2.0 / 11.0)
    want_grid = d * grid + (np.float32(1) - d) * grid1
    want_mlp = d * mlp + (np.float32(1) - d) * mlp1
    moved = grid1 != grid
    want_grid[~moved] = grid[~moved]
    Fq = random_features(rng, 1000, LO, HI)
    out = engine.cache_query(Fq)
    ref = forward_bf16(encode(Fq, want_grid, LO, HI)[0], want_mlp)
    assert_bf16_close(out, ref)
    live = forward_bf16(encode(Fq, grid1, LO, HI)[0], mlp1)
    assert np.abs(out - live).max() > 1e-3  # it is not the live network
    engine.set_cache_averaging(0.0)
    assert_bf16_close(engine.cache_query(Fq), live)
