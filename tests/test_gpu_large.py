"""Config 5 at full size (the largest run): a 19,999,980-triangle heightfield
plus 4,096 instanced 1,280-triangle icospheres (25.2 M triangles in the
scene), a 4096x2048 sky, 3840x2160. Checked through properties that do not
need a CPU render of the scene: the device BVH equals the host LBVH reference
byte for byte, every closest hit of a ray set is the nearest of all 25.2 M
world-space triangles (brute force in numpy), and a few samples of the 4K
frame accumulate to a finite, opaque image."""
import numpy as np
import pytest

from miniraytrace_b200 import abi, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def large_scene():
    return scenes.large()


def world_triangles(s):
    """All instanced triangles in world space, (N, 3, 3) float64, with the
    (instance position in s.instances, first triangle) of each instance."""
    tris, starts = [], []
    n = 0
    for mi, xf, _ in s.instances:
        m = s.meshes[mi]
        p = m.positions.astype(np.float64)
        if xf is not None:
            p = p @ xf[:, :3].T.astype(np.float64) + xf[:, 3].astype(np.float64)
        t = p[m.indices.reshape(-1, 3)]
        tris.append(t)
        starts.append(n)
        n += t.shape[0]
    return np.concatenate(tris), starts


def nearest_hits(tris, o, d):
    """Moeller-Trumbore over every triangle: (t of the nearest hit, its index,
    t of the second nearest) per ray, t in (1e-4, inf)."""
    v0 = tris[:, 0]
    e1 = tris[:, 1] - v0
    e2 = tris[:, 2] - v0
    out = []
    for k in range(o.shape[0]):
        p = np.cross(d[k], e2)
        det = np.einsum("ij,ij->i", e1, p)
        ok = np.abs(det) > 1e-18
        inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
        sv = o[k] - v0
        u = np.einsum("ij,ij->i", sv, p) * inv
        q = np.cross(sv, e1)
        v = (q @ d[k]) * inv
        t = np.einsum("ij,ij->i", e2, q) * inv
        hit = ok & (u >= 0) & (v >= 0) & (u + v <= 1) & (t > 1e-4)
        t = np.where(hit, t, np.inf)
        two = np.argpartition(t, 1)[:2]
        two = two[np.argsort(t[two])]
        out.append((t[two[0]], int(two[0]), t[two[1]]))
    return out


def test_large_scene_builds_traces_and_renders(gpu, large_scene):
    s = large_scene
    w, h = s.settings["width"], s.settings["height"]
    e = gpu.Engine(w, h)
    ids = s.apply(e)
    st = e.commit()
    assert st["blasRebuilt"] == 2
    stats = e.stats()
    assert stats["triangles"] == 19_999_980 + 1280 and stats["instances"] == 4097

    # the engine's device BVH of the big mesh is the host LBVH reference
    big = s.meshes[0]
    hn, ho = gpu.build_mesh_bvh(big.positions, big.indices, abi.MRTX_BVH_HOST_LBVH)
    dn, do = gpu.build_mesh_bvh(big.positions, big.indices, abi.MRTX_BVH_DEVICE_LBVH, engine=e)
    assert len(dn) == len(hn) and np.array_equal(do, ho) and dn.tobytes() == hn.tobytes()
    del hn, ho, dn, do

    # closest hits against brute force over all world-space triangles
    rng = np.random.default_rng(11)
    n = 24
    o = np.stack([rng.uniform(-0.9, 0.9, n), np.full(n, 0.6), rng.uniform(-0.9, 0.15, n)], 1)
    # aimed at points over the cropped terrain (z up to 0.19), plus two rays
    # that leave it and must miss everything
    target = np.stack([rng.uniform(-0.95, 0.95, n), np.zeros(n), rng.uniform(-0.95, 0.15, n)], 1)
    d = target - o
    d[-2:] = [[0.3, 0.05, 1.0], [-1.0, 0.02, 0.1]]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    hits = e.trace_rays(o.astype(np.float32), d.astype(np.float32))
    tris, starts = world_triangles(s)
    ref = nearest_hits(tris, o.astype(np.float32).astype(np.float64), d.astype(np.float32).astype(np.float64))
    inst_pos = {iid: k for k, iid in enumerate(ids["instances"])}
    checked = 0
    assert np.isinf(ref[-1][0]) and np.isinf(ref[-2][0])
    for k, (t_ref, tri_ref, t_second) in enumerate(ref):
        assert hits["hit"][k] == (1 if np.isfinite(t_ref) else 0), k
        if not np.isfinite(t_ref):
            continue
        assert abs(hits["t"][k] - t_ref) <= 1e-5 * t_ref + 1e-6, (k, hits["t"][k], t_ref)
        if t_second - t_ref > 1e-5 * t_ref:  # a unique nearest triangle
            tri_gpu = starts[inst_pos[int(hits["instance"][k])]] + int(hits["prim"][k])
            assert tri_gpu == tri_ref, k
            checked += 1
    assert checked >= n // 2
    assert sum(np.isfinite(r[0]) for r in ref) == n - 2

    # a few samples of the 4K frame
    e.render_frames(2)
    img = e.read_framebuffer(abi.MRT_PIXEL_RGBA32F_LINEAR)
    assert img.shape == (h, w, 4) and np.isfinite(img).all() and (img[..., 3] == 1.0).all()
    assert img[..., :3].mean() > 0.01
    e.close()
