"""Traversal parity (GPU, through the C ABI extension mrtxTraceRays).

Gate: closest-hit primitive ids bit-exact against the brute-force oracle
(Moeller-Trumbore over every triangle in original order, reference
tests/bvh_tests.cpp:145-151) on non-degenerate rays, t within 1e-6 relative.
A ray is non-degenerate when the oracle's hit has smallest barycentric
>= 1e-5 and the second-nearest accepted t differs by more than 1e-5 relative.
The GPU uses a watertight test (Woop et al. 2013), which may legitimately
differ from Moeller-Trumbore only on the excluded near-edge / near-tie rays.
"""
import os
from pathlib import Path

import numpy as np
import pytest

from miniraytrace_b200 import scenes

GOLDEN = Path(__file__).resolve().parent / "golden"
pytestmark = pytest.mark.gpu


def nondegenerate(bf, t2, mb):
    t = bf["t"]
    return (bf["hit"] == 1) & (mb >= 1e-5) & (np.abs(t2 - t) > 1e-5 * np.abs(t))


def check_parity(gh, bf, t2, mb, min_hits=50):
    nd = nondegenerate(bf, t2, mb)
    miss = bf["hit"] == 0
    assert nd.sum() >= min_hits
    assert (gh["hit"][nd] == 1).all()
    assert np.array_equal(gh["prim"][nd], bf["prim"][nd])
    assert np.array_equal(gh["instance"][nd], bf["instance"][nd])
    rel = np.abs(gh["t"][nd] - bf["t"][nd]) / np.abs(bf["t"][nd])
    assert rel.max() <= 1e-6, rel.max()
    # clear misses stay misses (a watertight hit may only appear on a near-edge ray)
    assert (gh["hit"][miss] == 0).mean() >= 0.999
    return nd.sum()


def soup(target, tris):
    pos = np.asarray(tris, np.float32).reshape(-1, 3)
    mesh = target.add_mesh(pos, np.arange(pos.shape[0], dtype=np.uint32))
    target.add_instance(mesh, None, 0)
    target.commit()


def test_bvh_tests_rays_vs_bruteforce(gpu, oracle_lib):
    g = np.load(GOLDEN / "bvh_cases.npz")
    e = gpu.Engine(16, 16)
    o = oracle_lib.OracleScene(16, 16)
    soup(e, g["tris7"])
    soup(o, g["tris7"])
    rays = g["rays123"]
    gh = e.trace_rays(rays[:, :3], rays[:, 3:])
    bf, t2, mb = o.trace_bruteforce(rays[:, :3], rays[:, 3:])
    check_parity(gh, bf, t2, mb)
    occ = e.trace_shadow_rays(rays[:, :3], rays[:, 3:])
    assert (occ[bf["hit"] == 0] == 0).mean() >= 0.999
    assert (occ[nondegenerate(bf, t2, mb)] == 1).all()
    e.close()


def test_dense_soup_many_rays(gpu, oracle_lib):
    rng = np.random.default_rng(11)
    n = 4000
    base = rng.uniform(-5, 5, (n, 3)).astype(np.float32)
    tris = np.concatenate([base, base + rng.uniform(-0.6, 0.6, (n, 3)), base + rng.uniform(-0.6, 0.6, (n, 3))], 1)
    e = gpu.Engine(16, 16)
    o = oracle_lib.OracleScene(16, 16)
    soup(e, tris)
    soup(o, tris)
    m = 20000
    org = rng.uniform(-8, 8, (m, 3)).astype(np.float32)
    d = rng.normal(size=(m, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    gh = e.trace_rays(org, d)
    bf, t2, mb = o.trace_bruteforce(org, d, threads=8)
    assert check_parity(gh, bf, t2, mb, min_hits=2000) > 2000
    e.close()


def test_instanced_scene_primary_rays(gpu, oracle_lib):
    """Box + sphere (config 1) and translated/scaled instances."""
    s = scenes.box_sphere(64, 64)
    pos, idx, nrm = scenes.icosphere(2)
    s.meshes.append(scenes.MeshSpec(pos, idx, nrm))
    for k, (x, y, z, r) in enumerate([(0.6, 1.4, -0.3, 0.2), (-0.5, 1.2, 0.4, 0.15), (0.2, 1.7, 0.5, 0.1)]):
        s.instances.append((len(s.meshes) - 1, np.array([[r, 0, 0, x], [0, r, 0, y], [0, 0, r, z]], np.float32), 0))
    e = gpu.Engine(64, 64)
    o = oracle_lib.OracleScene(64, 64)
    s.apply(e)
    s.apply(o)
    e.commit()
    o.commit()
    rng = np.random.default_rng(5)
    m = 30000
    org = np.tile(np.array([[0.0, 1.0, 3.6]], np.float32), (m, 1))
    d = np.stack([rng.uniform(-0.45, 0.45, m), rng.uniform(-0.5, 0.4, m), -np.ones(m)], 1).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    gh = e.trace_rays(org, d)
    bf, t2, mb = o.trace_bruteforce(org, d, threads=8)
    check_parity(gh, bf, t2, mb, min_hits=20000)
    # secondary rays from inside the box in all directions
    org2 = rng.uniform([-0.9, 0.1, -0.9], [0.9, 1.9, 0.9], (m, 3)).astype(np.float32)
    d2 = rng.normal(size=(m, 3)).astype(np.float32)
    d2 /= np.linalg.norm(d2, axis=1, keepdims=True)
    gh2 = e.trace_rays(org2, d2)
    bf2, t22, mb2 = o.trace_bruteforce(org2, d2, threads=8)
    check_parity(gh2, bf2, t22, mb2, min_hits=20000)
    e.close()


def test_heightfield_rays(gpu, oracle_lib):
    pos, idx, nrm, _ = scenes.heightfield(96)
    e = gpu.Engine(16, 16)
    o = oracle_lib.OracleScene(16, 16)
    for t in (e, o):
        mesh = t.add_mesh(pos, idx, nrm)
        t.add_instance(mesh, None, 0)
        t.commit()
    rng = np.random.default_rng(9)
    m = 20000
    org = np.stack([rng.uniform(-1, 1, m), np.full(m, 0.8), rng.uniform(-1, 1, m)], 1).astype(np.float32)
    d = np.stack([rng.uniform(-0.6, 0.6, m), -np.ones(m), rng.uniform(-0.6, 0.6, m)], 1).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    gh = e.trace_rays(org, d)
    bf, t2, mb = o.trace_bruteforce(org, d, threads=8)
    check_parity(gh, bf, t2, mb, min_hits=10000)
    e.close()


def test_empty_scene_and_tmax(gpu):
    e = gpu.Engine(8, 8)
    gh = e.trace_rays(np.zeros((4, 3)), np.tile([[0, 0, -1.0]], (4, 1)))
    assert (gh["hit"] == 0).all()
    tri = np.array([[-1, -1, -2], [1, -1, -2], [0, 1, -2]], np.float32)
    soup(e, tri)
    gh = e.trace_rays(np.zeros((3, 3)), np.tile([[0, 0, -1.0]], (3, 1)), t_max=np.float32(5.0))
    assert (gh["hit"] == 1).all() and np.allclose(gh["t"], 2.0)
    gh = e.trace_rays(np.zeros((1, 3)), [[0, 0, -1.0]], t_max=1.5)
    assert gh["hit"][0] == 0
    occ = e.trace_shadow_rays(np.zeros((2, 3)), [[0, 0, -1.0], [0, 0, 1.0]])
    assert list(occ) == [1, 0]
    e.close()


def camera_rays(cam, width, height, n, rng):
    """Jittered primary rays of the scene camera through n random pixels, in
    pixel order (as a wave's first bounce holds them)."""
    pos = np.asarray(cam["position"], np.float64)
    fwd = np.asarray(cam["target"], np.float64) - pos
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, np.asarray(cam["up"], np.float64))
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    th = np.tan(np.radians(cam["fov_y_deg"]) * 0.5)
    pix = np.sort(rng.choice(width * height, n, replace=False))
    u = (pix % width + rng.uniform(0, 1, n)) / width
    v = (pix // width + rng.uniform(0, 1, n)) / height
    sx = th * width / height * (2 * u - 1)
    sy = th * (1 - 2 * v)
    d = fwd + sx[:, None] * right + sy[:, None] * up
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.tile(pos.astype(np.float32), (n, 1)), d.astype(np.float32)


def test_wavefront_extend_kernel_at_config2_scale(gpu, oracle_lib):
    """The renderer's own closest-hit stage (waveExtendKernel: persistent
    warps, lane refill, warp-batched triangle tests) on the 2,420,738-triangle
    config-2 scene: 262,144 primary and secondary rays give hits identical
    to the one-ray-per-thread query kernel, and a 3,000-ray sample (2,500
    hits, 500 misses) matches the brute-force oracle (ids bit-exact on non-degenerate rays, t within
    1e-6 relative)."""
    s = scenes.terrain()
    W, H = s.settings["width"], s.settings["height"]
    e = gpu.Engine(W, H)
    s.apply(e)
    e.commit()
    rng = np.random.default_rng(21)
    n = 131072
    o1, d1 = camera_rays(s.camera, W, H, n, rng)
    h1 = e.trace_rays(o1, d1, wavefront=True)
    # secondary rays from the primary hits, in all directions, mostly upward
    hit = h1["hit"] == 1
    assert hit.mean() > 0.2  # the camera sees a third terrain, two thirds sky
    p = o1[hit] + h1["t"][hit][:, None] * d1[hit]
    k = p.shape[0]
    d2 = rng.normal(size=(k, 3)).astype(np.float32)
    d2[:, 1] = np.where(rng.uniform(size=k) < 0.8, np.abs(d2[:, 1]), d2[:, 1])
    d2 /= np.linalg.norm(d2, axis=1, keepdims=True)
    o2 = (p + np.float32(1e-3) * np.array([0, 1, 0], np.float32)).astype(np.float32)
    take = rng.choice(k, min(k, n), replace=False)
    org = np.concatenate([o1, o2[take]]).astype(np.float32)
    dirs = np.concatenate([d1, d2[take]]).astype(np.float32)
    wave = e.trace_rays(org, dirs, wavefront=True)
    single = e.trace_rays(org, dirs)
    for f in ("hit", "prim", "instance", "t", "u", "v"):
        assert np.array_equal(wave[f], single[f]), f
    o = oracle_lib.OracleScene(W, H)
    s.apply(o)
    o.commit()
    # 2,500 of the rays the kernel reports as hits (primary and secondary
    # alike) and 500 it reports as misses: two thirds of the camera's rays see
    # sky, and a brute-force hit among the misses would be a kernel miss
    hits = np.flatnonzero(wave["hit"] == 1)
    misses = np.flatnonzero(wave["hit"] == 0)
    sample = np.concatenate([rng.choice(hits, 2500, replace=False), rng.choice(misses, 500, replace=False)])
    bf, t2, mb = o.trace_bruteforce(org[sample], dirs[sample], threads=os.cpu_count() or 8)
    got = check_parity(wave[sample], bf, t2, mb, min_hits=2000)
    print(f"wavefront extend kernel: {got} non-degenerate rays bit-exact against brute force")
    e.close()
