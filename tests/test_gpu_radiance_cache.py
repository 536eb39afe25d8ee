"""Radiance cache network on the GPU against a numpy implementation of the
same network: hash-grid + spherical-harmonics encoding and 5 x 64 ReLU MLP
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

pytestmark = pytest.mark.gpu

LEVELS, T = 16, 1 << 19
SCALES = np.array([16.0 * 2.0 ** (l * 7.0 / 15.0) for l in range(LEVELS)], np.float32)
LR = 1e-2


def grid_index(x, y, z, res):
    if (res + 1) ** 3 <= T:
        return x + (res + 1) * (y + (res + 1) * z)
    return ((x * np.uint64(1)) ^ (y * np.uint64(2654435761)) ^ (z * np.uint64(805459861))) & np.uint64(T - 1)


def sh4(d):
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    xx, yy, zz = x * x, y * y, z * z
    return np.stack([
        np.full_like(x, 0.28209479177387814), -0.48860251190291987 * y, 0.48860251190291987 * z,
        -0.48860251190291987 * x, 1.0925484305920792 * x * y, -1.0925484305920792 * y * z,
        0.94617469575755997 * zz - 0.31539156525251999, -1.0925484305920792 * x * z,
        0.54627421529603959 * (xx - yy), 0.59004358992664352 * y * (-3 * xx + yy), 2.8906114426405538 * x * y * z,
        0.45704579946446572 * y * (1 - 5 * zz), 0.3731763325901154 * z * (5 * zz - 3),
        0.45704579946446572 * x * (1 - 5 * zz), 1.4453057213202769 * z * (xx - yy),
        0.59004358992664352 * x * (-xx + 3 * yy)], 1)


def encode(F, grid, lo, hi):
    """(n, 64) encoding and, per level, the 8 corner indices and weights."""
    n = F.shape[0]
    inv = (np.float32(1.0) / (hi - lo)).astype(np.float32)
    p = np.clip((F[:, :3] - lo) * inv, 0, 1).astype(np.float32)
    enc = np.zeros((n, 64), np.float64)
    g2 = grid.reshape(-1, 2).astype(np.float64)
    corners = []
    for l in range(LEVELS):
        s = SCALES[l]
        res = int(np.ceil(s))
        x = (p * s).astype(np.float32)
        fl = np.minimum(np.floor(x), np.float32(res - 1))
        b = fl.astype(np.uint64)
        fr = (x - fl).astype(np.float64)
        lvl = []
        for c in range(8):
            o = [(c >> a) & 1 for a in range(3)]
            w = np.ones(n)
            for a in range(3):
                w = w * (fr[:, a] if o[a] else 1 - fr[:, a])
            idx = np.uint64(l * T) + grid_index(b[:, 0] + np.uint64(o[0]), b[:, 1] + np.uint64(o[1]),
                                                b[:, 2] + np.uint64(o[2]), res)
            idx = idx.astype(np.int64)
            enc[:, 2 * l] += w * g2[idx, 0]
            enc[:, 2 * l + 1] += w * g2[idx, 1]
            lvl.append((idx, w))
        corners.append(lvl)
    d = F[:, 3:6].astype(np.float64)
    d = d / np.sqrt(np.maximum((d * d).sum(1, keepdims=True), 1e-20))
    enc[:, 32:48] = sh4(d)
    enc[:, 48:51] = 0.5 * F[:, 6:9] + 0.5
    enc[:, 51] = F[:, 9]
    enc[:, 52:55] = F[:, 10:13]
    enc[:, 55] = 1.0
    return enc, corners


def forward(enc, mlp):
    W = mlp.reshape(6, 64, 64).astype(np.float64)
    hs = [enc]
    h = enc
    for l in range(5):
        h = np.maximum(h @ W[l].T, 0.0)
        hs.append(h)
    return h @ W[5][:3].T, hs


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    b = np.asarray(x, np.float64).astype(np.float32).view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def assert_bf16_close(out, ref, msg=""):
    near = np.isclose(out, ref, rtol=5e-3, atol=2e-4)
    assert near.mean() >= 0.999, (msg, near.size - near.sum())
    np.testing.assert_allclose(out, ref, rtol=1e-2, atol=2e-3, err_msg=msg)


def forward_bf16(enc, mlp):
    """The tensor-core inference: BF16 operands, FP32 (here FP64) sums."""
    W = bf16(mlp).reshape(6, 64, 64)
    h = bf16(enc)
    for l in range(5):
        h = bf16(np.maximum(h @ W[l].T, 0.0))
    return np.maximum(h @ W[5][:3].T, 0.0)


def gradients(F, targets, grid, mlp, lo, hi):
    """Gradients of the mean relative L2 loss (denominator held fixed) as the
    tensor-core training step forms them: the encoding, weights, hidden
    activations and each back-propagated gradient rounded to BF16."""
    enc, corners = encode(F, grid, lo, hi)
    W = bf16(mlp).reshape(6, 64, 64)
    hs = [bf16(enc)]
    for l in range(5):
        hs.append(bf16(np.maximum(hs[-1] @ W[l].T, 0.0)))
    y = hs[5] @ W[5][:3].T
    n = F.shape[0]
    dz = bf16(2.0 * (y - targets) / (y * y + 0.01) / (3.0 * n))
    gW = np.zeros((6, 64, 64))
    gW[5][:3] = dz.T @ hs[5]
    delta = dz @ W[5][:3]
    for l in range(4, -1, -1):
        delta = bf16(delta * (hs[l + 1] > 0))
        gW[l] = delta.T @ hs[l]
        delta = delta @ W[l]
    gG = np.zeros(grid.size)
    for l in range(LEVELS):
        for idx, w in corners[l]:
            np.add.at(gG, 2 * idx, w * delta[:, 2 * l])
            np.add.at(gG, 2 * idx + 1, w * delta[:, 2 * l + 1])
    return gW.ravel(), gG


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
    gW, gG = gradients(F, targets.astype(np.float64), grid, mlp, LO, HI)
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
