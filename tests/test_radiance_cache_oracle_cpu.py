"""Pins the radiance-cache oracle (oracle/radiance_cache.py) before the GPU
tests trust it: its FP64 gradients of the relative L2 loss (denominator held
fixed at the evaluation point) equal central finite differences of the loss,
for weights of every layer (step 1e-6) and for hash-grid entries of coarse
(dense) and fine (hashed) levels (step 1e-4), within 1e-5 relative + 1e-10
absolute. Also checks that
the BF16-emulating gradients agree in sign with the FP64 ones where the
latter are large, and the BF16 rounding against torch's."""
import numpy as np
import pytest

from oracle import radiance_cache as rc

LO = np.array([-2.0, 0.0, 1.0], np.float32)
HI = np.array([3.0, 4.0, 2.5], np.float32)


def setup(n=48, seed=9):
    rng = np.random.default_rng(seed)
    F = np.zeros((n, 16), np.float32)
    F[:, :3] = rng.uniform(LO, HI, (n, 3))
    d = rng.normal(size=(n, 3))
    F[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    nn = rng.normal(size=(n, 3))
    F[:, 6:9] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    F[:, 9] = rng.uniform(0, 1, n)
    F[:, 10:13] = rng.uniform(0, 1, (n, 3))
    grid = rng.normal(size=16 * (1 << 19) * 2) * 0.5
    mlp = rng.uniform(-1, 1, 6 * 64 * 64) * np.sqrt(6.0 / 128)
    mlp.reshape(6, 64, 64)[5][3:] = 0
    targets = rng.uniform(0, 2, (n, 3))
    return F, grid, mlp, targets


def loss_at(F, targets, grid, mlp, den):
    y = rc.forward(rc.encode(F, grid, LO, HI)[0], mlp)[0]
    return rc.relative_l2_loss(y, targets, den)


def test_fp64_gradients_equal_finite_differences():
    F, grid, mlp, targets = setup()
    y0 = rc.forward(rc.encode(F, grid, LO, HI)[0], mlp)[0]
    den = y0 * y0 + 0.01
    gW, gG = rc.gradients_fp64(F, targets, grid, mlp, LO, HI)
    rng = np.random.default_rng(1)
    h = 1e-6
    # weights: the largest entries of each layer's gradient plus random ones
    picks = []
    for l in range(6):
        layer = np.arange(l * 4096, (l + 1) * 4096)
        rows = 3 * 64 if l == 5 else 4096
        g = np.abs(gW[layer[:rows]])
        picks += list(layer[np.argsort(-g)[:4]]) + list(rng.choice(layer[:rows], 2, replace=False))
    for k in picks:
        p, m = mlp.copy(), mlp.copy()
        p[k] += h
        m[k] -= h
        fd = (loss_at(F, targets, grid, p, den) - loss_at(F, targets, grid, m, den)) / (2 * h)
        assert abs(fd - gW[k]) <= 1e-5 * abs(gW[k]) + 1e-10, (k, fd, gW[k])
    # grid entries the samples touch: level 0 (dense) and level 15 (hashed)
    touched = np.nonzero(gG)[0]
    coarse = touched[touched < 2 * (1 << 19)]
    fine = touched[touched >= 2 * 15 * (1 << 19)]
    assert len(coarse) > 10 and len(fine) > 10
    # (a larger step: grid gradients are small next to the loss, and below
    # 1e-5 the difference quotient is dominated by the loss's rounding)
    hg = 1e-4
    for k in list(rng.choice(coarse, 8, replace=False)) + list(rng.choice(fine, 8, replace=False)):
        p, m = grid.copy(), grid.copy()
        p[k] += hg
        m[k] -= hg
        fd = (loss_at(F, targets, p, mlp, den) - loss_at(F, targets, m, mlp, den)) / (2 * hg)
        assert abs(fd - gG[k]) <= 1e-5 * abs(gG[k]) + 1e-10, (k, fd, gG[k])


def test_bf16_gradients_follow_fp64_signs():
    F, grid, mlp, targets = setup(n=256, seed=4)
    gW, gG = rc.gradients_fp64(F, targets, grid, mlp, LO, HI)
    bW, bG = rc.gradients_bf16(F, targets, grid, mlp, LO, HI)
    for g, b in ((gW, bW), (gG, bG)):
        big = np.abs(g) > 0.05 * np.abs(g).max()
        assert big.sum() > 50
        assert (np.sign(b[big]) == np.sign(g[big])).mean() >= 0.99


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    x = np.random.default_rng(2).normal(size=100000) * np.exp(np.random.default_rng(3).uniform(-20, 20, 100000))
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).double().numpy()
    assert np.array_equal(rc.bf16(x), ref)
