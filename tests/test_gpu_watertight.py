"""Watertightness and degenerate geometry (GPU, through mrtxTraceRays and the
render path).

- A closed icosphere is hit by every ray aimed exactly at one of its
  vertices, edge midpoints or face centroids, from its centre and from
  three outside points: no ray slips through a shared vertex or edge (the
  reason for the watertight test of Woop et al. 2013), and every shadow ray
  from the centre is occluded.
- Zero-area triangles (two equal corners, collinear corners, one point)
  mixed into a random soup change nothing: closest hits equal the
  brute-force oracle's on non-degenerate rays, as in test_gpu_trace.py.
- Zero bounces (direct light only) and the bounce cap of 16 render at
  parity with the oracle (99.9% of pixels within 1e-3).
"""
import numpy as np
import pytest

from miniraytrace_b200 import abi, scenes

from test_gpu_render import parity_fraction, render_both
from test_gpu_trace import check_parity, soup

pytestmark = pytest.mark.gpu


def surface_points(pos, idx):
    tri = idx.reshape(-1, 3)
    edges = np.sort(np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]]), axis=1)
    edges = np.unique(edges, axis=0)
    mids = (pos[edges[:, 0]] + pos[edges[:, 1]]) * 0.5
    cents = pos[tri].mean(axis=1)
    return np.concatenate([pos, mids, cents]).astype(np.float64)


def test_no_ray_slips_through_shared_vertices_or_edges(gpu):
    pos, idx, _ = scenes.icosphere(4)  # closed, 5,120 triangles, vertices on the unit sphere
    pos = np.asarray(pos, np.float32)
    e = gpu.Engine(16, 16)
    e.add_instance(e.add_mesh(pos, idx), None, 0)
    e.commit()
    pts = surface_points(pos.astype(np.float64), idx)
    # from the centre
    d = (pts / np.linalg.norm(pts, axis=1, keepdims=True)).astype(np.float32)
    o = np.zeros_like(d)
    gh = e.trace_rays(o, d)
    assert (gh["hit"] == 1).all(), int((gh["hit"] == 0).sum())
    assert (gh["t"] > 0.99).all() and (gh["t"] <= 1.0 + 1e-5).all()
    assert (e.trace_shadow_rays(o, d) == 1).all()
    # from outside, aimed at the points facing the origin (cosine >= 0.2, so a
    # direction rounded to float32 cannot pass beside the silhouette): the ray
    # enters the convex surface at the point it was aimed at
    for origin in ((3.0, 2.0, 5.0), (-4.0, 1.0, -2.0), (0.5, -6.0, 0.25)):
        org = np.array(origin, np.float64)
        to_o = org - pts
        dist = np.linalg.norm(to_o, axis=1)
        facing = np.einsum("ij,ij->i", pts / np.linalg.norm(pts, axis=1, keepdims=True), to_o) / dist >= 0.2
        q, dq = pts[facing], dist[facing]
        assert len(q) > 2000
        d = ((q - org) / dq[:, None]).astype(np.float32)
        gh = e.trace_rays(np.tile(np.array(origin, np.float32), (len(d), 1)), d)
        assert (gh["hit"] == 1).all(), (origin, int((gh["hit"] == 0).sum()))
        assert (np.abs(gh["t"] - dq) <= 1e-5 * dq).all()
    e.close()


def test_degenerate_triangles_among_normal_ones(gpu, oracle_lib):
    rng = np.random.default_rng(21)
    good = rng.uniform(-1, 1, (600, 3, 3))
    a = rng.uniform(-1, 1, (200, 1, 3))
    two_equal = np.concatenate([a, a, rng.uniform(-1, 1, (200, 1, 3))], axis=1)
    p0, p1 = rng.uniform(-1, 1, (2, 200, 1, 3))
    collinear = np.concatenate([p0, p1, 0.3 * p0 + 0.7 * p1], axis=1)
    point = np.repeat(rng.uniform(-1, 1, (50, 1, 3)), 3, axis=1)
    tris = np.concatenate([good, two_equal, collinear, point])
    tris = tris[rng.permutation(len(tris))]
    e = gpu.Engine(16, 16)
    o = oracle_lib.OracleScene(16, 16)
    soup(e, tris)
    soup(o, tris)
    # from outside the soup (a sphere of radius 4) towards points inside it, so
    # hit distances are not tiny (the t tolerance is relative)
    u = rng.normal(size=(4000, 3))
    org = (4.0 * u / np.linalg.norm(u, axis=1, keepdims=True)).astype(np.float32)
    d = rng.uniform(-1, 1, (4000, 3)) - org
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    gh = e.trace_rays(org, d)
    bf, t2, mb = o.trace_bruteforce(org, d)
    assert check_parity(gh, bf, t2, mb, min_hits=500) >= 500
    e.close()


@pytest.mark.parametrize("bounces", [0, 16])
def test_bounce_extremes_parity(gpu, oracle_lib, bounces):
    s = scenes.box_sphere(64, 64)
    s.settings["max_bounces"] = bounces
    e, img, ref, _ = render_both(gpu, oracle_lib, s, 4)
    assert np.isfinite(img).all() and (img[..., 3] == 1.0).all()
    assert parity_fraction(img, ref) >= 0.999
    e.close()
