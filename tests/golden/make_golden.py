"""Regenerates the golden fixtures in this directory (run from the repo root:
``python tests/golden/make_golden.py``). Needs g++ and the reference checkout
(for oracle/_ref/libref_bvh.so, the reference's own BVH builder).

Fixtures:
  bvh_cases.npz  -- the triangle/ray sets of reference tests/bvh_tests.cpp
                    (via gen_bvh_cases.cpp) and, for each triangle set, the
                    BVH2 nodes and primOrder that the reference's
                    BvhBuilder::build(bounds, 4) produces;
  pcg4d.npz      -- pcg4d outputs for 64 seeded states, computed from the
                    published pcg4d recurrence (Jarzynski & Olano 2020, as in
                    reference random.glsl:6-12) in numpy uint32 arithmetic;
  env_cdf.npz    -- a 64 x 32 procedural sky and the CDF + integral that the
                    oracle's restatement of Renderer.cpp:620-655 gives (kept to
                    detect drift in the oracle; the renderer code itself cannot
                    be compiled here).
"""
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))


def tri_aabbs(t):
    t = t.reshape(-1, 3, 3)
    return np.concatenate([t.min(1), t.max(1)], 1).astype(np.float32)


def pcg4d_np(v):
    v = v.astype(np.uint64)
    m = np.uint64(0xFFFFFFFF)
    v = (v * np.uint64(1664525) + np.uint64(1013904223)) & m
    x, y, z, w = v[:, 0].copy(), v[:, 1].copy(), v[:, 2].copy(), v[:, 3].copy()
    x = (x + y * w) & m; y = (y + z * x) & m; z = (z + x * y) & m; w = (w + y * z) & m
    x ^= x >> np.uint64(16); y ^= y >> np.uint64(16); z ^= z >> np.uint64(16); w ^= w >> np.uint64(16)
    x = (x + y * w) & m; y = (y + z * x) & m; z = (z + x * y) & m; w = (w + y * z) & m
    return np.stack([x, y, z, w], 1).astype(np.uint32)


def main():
    import oracle
    from oracle import build_oracle
    build_oracle.build()
    with tempfile.TemporaryDirectory() as td:
        exe = Path(td) / "gen"
        subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe), str(HERE / "gen_bvh_cases.cpp")], check=True)
        f = [Path(td) / n for n in ("t42.bin", "t7.bin", "r123.bin")]
        subprocess.run([str(exe), *map(str, f)], check=True)
        t42 = np.fromfile(f[0], np.float32).reshape(-1, 9)
        t7 = np.fromfile(f[1], np.float32).reshape(-1, 9)
        r123 = np.fromfile(f[2], np.float32).reshape(-1, 6)
    n42, o42 = oracle.bvh_build(tri_aabbs(t42), 4, use_reference=True)
    n7, o7 = oracle.bvh_build(tri_aabbs(t7), 4, use_reference=True)
    np.savez_compressed(HERE / "bvh_cases.npz", tris42=t42, tris7=t7, rays123=r123,
                        nodes42=n42.view(np.uint32).reshape(-1, 8), order42=o42,
                        nodes7=n7.view(np.uint32).reshape(-1, 8), order7=o7)
    rng = np.random.default_rng(2020)
    states = rng.integers(0, 2**32, size=(64, 4), dtype=np.uint64).astype(np.uint32)
    states[:8] = [[0, 0, 0, 1], [1, 2, 3, 4], [255, 255, 0, 1], [0, 0, 15, 3], [1919, 1079, 63, 40],
                  [4294967295, 0, 1, 2], [7, 7, 7, 7], [128, 64, 1023, 12]]
    np.savez_compressed(HERE / "pcg4d.npz", states=states, out=pcg4d_np(states))
    from miniraytrace_b200 import scenes
    sky = scenes.procedural_sky(64, 32, sun_sigma_deg=6.0, sun_peak=50.0)
    cdf, integral = oracle.env_cdf(sky)
    np.savez_compressed(HERE / "env_cdf.npz", sky=sky, cdf=cdf, integral=np.float32(integral))
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))


if __name__ == "__main__":
    main()
