"""ORACLE -- test infrastructure only. Not part of the product.

CPU restatement (numpy) of the radiance-cache network of
miniraytrace_b200/csrc/cuda/radiance_cache.cu, the checker its GPU tests
compare against. The reference has no radiance cache; this restates the
published methods the kernels implement (the multiresolution hash encoding of
Mueller et al. 2022 with its spatial hash and geometric level scales, degree-4
real spherical harmonics, and the 5 x 64 ReLU network with the relative L2
loss of Mueller et al. 2021), in FP64, plus variants that round to BF16 where
the tensor-core kernels do.

Pinned by tests/test_radiance_cache_oracle_cpu.py: the FP64 gradients equal
central finite differences of the loss.

Features: 16 floats per query (position, outgoing direction, normal,
roughness, albedo rgb, unused). Encoding: 64 values (16 levels x 2 grid
features, 16 SH coefficients, normal mapped to [0, 1], roughness, albedo, a
constant 1, zero padding). Weights: 6 x 64 x 64 row-major (W5 uses rows 0..2).
"""
import numpy as np

LEVELS, T = 16, 1 << 19
SCALES = np.array([16.0 * 2.0 ** (l * 7.0 / 15.0) for l in range(LEVELS)], np.float32)


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


def forward_bf16(enc, mlp):
    """The tensor-core inference: BF16 operands, FP32 (here FP64) sums."""
    W = bf16(mlp).reshape(6, 64, 64)
    h = bf16(enc)
    for l in range(5):
        h = bf16(np.maximum(h @ W[l].T, 0.0))
    return np.maximum(h @ W[5][:3].T, 0.0)


def gradients_bf16(F, targets, grid, mlp, lo, hi):
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


def relative_l2_loss(y, targets, den):
    """Mean over samples and channels of (y - t)^2 / den, den = y0^2 + 0.01
    taken at the point the gradient is evaluated (held fixed)."""
    return float(np.mean((y - targets) ** 2 / den))


def gradients_fp64(F, targets, grid, mlp, lo, hi):
    """Exact FP64 gradients of the mean relative L2 loss with its
    denominator held fixed: (mlp gradient, grid gradient), both flat."""
    enc, corners = encode(F, grid, lo, hi)
    y, hs = forward(enc, mlp)
    W = mlp.reshape(6, 64, 64).astype(np.float64)
    n = F.shape[0]
    delta_out = 2.0 * (y - targets) / (y * y + 0.01) / (3.0 * n)
    gW = np.zeros((6, 64, 64))
    gW[5][:3] = delta_out.T @ hs[5]
    delta = delta_out @ W[5][:3]
    for l in range(4, -1, -1):
        delta = delta * (hs[l + 1] > 0)
        gW[l] = delta.T @ hs[l]
        delta = delta @ W[l]
    gG = np.zeros(grid.size)
    for l in range(LEVELS):
        for idx, w in corners[l]:
            np.add.at(gG, 2 * idx, w * delta[:, 2 * l])
            np.add.at(gG, 2 * idx + 1, w * delta[:, 2 * l + 1])
    return gW.ravel(), gG
