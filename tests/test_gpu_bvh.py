"""Device BVH builder: the GPU's LBVH + SAH-optimal collapse must equal the
host reference of the same algorithm byte for byte (nodes and triangle
order), and the engine renders with it (large meshes use it on commit)."""
import numpy as np
import pytest

from miniraytrace_b200 import abi

from test_wide_bvh_cpu import boxes_as_triangles, heightfield_mesh, soup_mesh

pytestmark = pytest.mark.gpu


def meshes():
    one = (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]], np.uint32))
    same = (one[0], np.tile(one[1], (50, 1)))
    flat = heightfield_mesh(30, 5)
    flat[0][:, 1] = 0.0
    rng = np.random.default_rng(5)
    c = rng.uniform(-5, 5, (3000, 3))
    r = rng.exponential(1.0, (3000, 1)) * rng.uniform(0.2, 1.0, (3000, 3))
    boxes = np.concatenate([c - r, c + r], 1)
    boxes[100:120] = boxes[0]
    return {"one": one, "two": soup_mesh(2, 1), "three": soup_mesh(3, 1), "same": same, "flat": flat,
            "soup": soup_mesh(5000, 7), "heightfield": heightfield_mesh(300, 9),
            "instances": boxes_as_triangles(boxes)}


@pytest.mark.parametrize("leaf", [3, 1])
@pytest.mark.parametrize("name", ["one", "two", "three", "same", "flat", "soup", "heightfield", "instances"])
def test_device_lbvh_equals_host(gpu, name, leaf):
    """Leaves of up to 3 triangles (meshes) and of one primitive (the
    instance tree, whose boxes enter the builder as degenerate triangles)."""
    pos, idx = meshes()[name]
    e = gpu.Engine(16, 16)
    hn, ho = gpu.build_mesh_bvh(pos, idx, abi.MRTX_BVH_HOST_LBVH, max_leaf_prims=leaf)
    dn, do = gpu.build_mesh_bvh(pos, idx, abi.MRTX_BVH_DEVICE_LBVH, max_leaf_prims=leaf, engine=e)
    # twice: the builder reuses its scratch
    dn2, do2 = gpu.build_mesh_bvh(pos, idx, abi.MRTX_BVH_DEVICE_LBVH, max_leaf_prims=leaf, engine=e)
    e.close()
    assert len(dn) == len(hn)
    assert np.array_equal(do, ho)
    assert dn.tobytes() == hn.tobytes()
    assert dn2.tobytes() == hn.tobytes() and np.array_equal(do2, ho)


def test_device_built_scene_renders_like_host_built(gpu):
    """A terrain of 44,402 triangles under 2,500 overlapping icosphere
    instances: by default the heightfield's BVH and the instance tree are
    built on the GPU (mrtxStats.commitDeviceBlas / commitDeviceTlas); an
    engine told to build both on the host (binned SAH) traces different
    trees over the same primitives, so closest hits (ids, and t to the bit)
    and the image must agree. Ties at shared edges may pick either
    triangle, so ids are gated at 99.9% of rays; t is gated on every ray."""
    from miniraytrace_b200 import scenes
    s = scenes.terrain(96, 64, spp=4, grid=150, spheres=2500, sky=(256, 128))
    engines = []
    for host in (False, True):
        e = gpu.Engine(96, 64)
        if host:
            e.set_bvh_build_thresholds(0xFFFFFFFF, 0xFFFFFFFF)
        ids = s.apply(e)
        e.commit()
        st = e.stats()
        assert (st["commitDeviceBlas"], st["commitDeviceTlas"]) == ((0, 0) if host else (1, 1)), st
        assert st["instances"] == 2501
        # an instance moved: the next commit rebuilds only the instance tree
        xf = np.array([[0.05, 0, 0, 0.1], [0, 0.05, 0, 0.3], [0, 0, 0.05, -0.2]], np.float32)
        e.set_instance_transform(ids["instances"][7], xf)
        e.commit()
        st2 = e.stats()
        assert (st2["commitDeviceBlas"], st2["commitDeviceTlas"]) == (0, 0 if host else 1), st2
        print(f"{'host' if host else 'device'} build: {st['commitBvhMs']:.2f} ms for the scene's BVHs, "
              f"{st2['commitBvhMs']:.2f} ms for the instance tree alone")
        engines.append(e)
    rng = np.random.default_rng(3)
    n = 20000
    org = np.tile(np.array([[0.0, 0.55, 2.1]], np.float32), (n, 1))
    # camera rays that land on the heightfield's [-1, 1]^2 footprint
    d = np.stack([rng.uniform(-0.3, 0.3, n), rng.uniform(-0.48, -0.2, n), -np.ones(n)], 1)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    hd, hh = (e.trace_rays(org, d) for e in engines)
    hw = engines[0].trace_rays(org, d, wavefront=True)
    assert np.array_equal(hd["hit"], hh["hit"]) and np.array_equal(hw["hit"], hh["hit"])
    m = hh["hit"] == 1
    assert m.mean() > 0.8, m.mean()
    assert np.array_equal(hd["t"][m], hh["t"][m]) and np.array_equal(hw["t"][m], hh["t"][m])
    same = (hd["prim"] == hh["prim"]) & (hd["instance"] == hh["instance"])
    assert same[m].mean() >= 0.999, same[m].mean()
    imgs = []
    for e in engines:
        for _ in range(4):
            e.render_frame()
        imgs.append(e.read_framebuffer(abi.MRT_PIXEL_RGBA32F_LINEAR))
        e.close()
    a, b = imgs
    exact = (a == b).all(-1).mean()
    close = (np.abs(a[..., :3] - b[..., :3]) <= 1e-3 * np.abs(b[..., :3]) + 1e-6).all(-1).mean()
    print(f"device-built vs host-built trees: {exact * 100:.3f}% of pixels bit-identical, {close * 100:.3f}% within 1e-3")
    assert np.isfinite(a).all() and close >= 0.999
