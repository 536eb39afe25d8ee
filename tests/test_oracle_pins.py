"""Pins the CPU oracle before it is trusted as the checker.

- BVH: the oracle's restated builder must produce exactly the nodes and
  primitive order of the reference's own BvhBuilder (core/src/accel/Bvh.cpp,
  compiled from its sources into oracle/_ref), on the input sets of the
  reference's tests/bvh_tests.cpp (fixtures) and on fresh random sets.
- The reference's BVH tests (topology, traversal == brute force, degenerate
  inputs: bvh_tests.cpp:91-188) are restated against the oracle.
- pcg4d golden vectors; environment-CDF fixture and properties.
- The reference's 2-instance TLAS leaves, of which its traversal enters
  only the first instance, and the oracle's switches around them (walk every
  leaf instance; brute force), on the room and an instanced terrain.
"""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def tri_aabbs(t):
    t = np.asarray(t, np.float32).reshape(-1, 3, 3)
    return np.concatenate([t.min(1), t.max(1)], 1)


@pytest.fixture(scope="module")
def cases():
    return np.load(GOLDEN / "bvh_cases.npz")


@pytest.mark.parametrize("key", ["42", "7"])
def test_oracle_bvh_equals_reference_fixture(oracle_lib, cases, key):
    nodes, order = oracle_lib.bvh_build(tri_aabbs(cases["tris" + key]), 4)
    assert np.array_equal(nodes.view(np.uint32).reshape(-1, 8), cases["nodes" + key])
    assert np.array_equal(order, cases["order" + key])


@pytest.mark.parametrize("seed,n,leaf", [(1, 1, 4), (2, 3, 4), (3, 1000, 4), (4, 3000, 1), (5, 20000, 4)])
def test_oracle_bvh_equals_reference_build(oracle_lib, seed, n, leaf):
    if oracle_lib.load_ref_bvh() is None:
        pytest.skip("reference BVH library not built (reference checkout absent)")
    rng = np.random.default_rng(seed)
    lo = rng.uniform(-50, 50, (n, 3)).astype(np.float32)
    hi = lo + rng.exponential(1.0, (n, 3)).astype(np.float32)
    if n > 100:  # include exact duplicates and flat boxes
        hi[:10] = lo[:10]
        lo[10:20] = lo[0]
        hi[10:20] = hi[0]
    ab = np.concatenate([lo, hi], 1)
    a_nodes, a_order = oracle_lib.bvh_build(ab, leaf)
    b_nodes, b_order = oracle_lib.bvh_build(ab, leaf, use_reference=True)
    assert a_nodes.tobytes() == b_nodes.tobytes()
    assert np.array_equal(a_order, b_order)


def test_bvh_topology(oracle_lib, cases):
    """bvh_tests.cpp:91-119: every primitive exactly once, children in range."""
    nodes, order = oracle_lib.bvh_build(tri_aabbs(cases["tris42"]), 4)
    n = cases["tris42"].shape[0]
    assert order.size == n and len(nodes) > 0
    seen = np.zeros(n, np.int64)
    leaf_prims = 0
    for nd in nodes:
        count = int(nd["packed"]) >> 2
        if count == 0:
            assert int(nd["leftOrPrim"]) + 1 < len(nodes)
        else:
            leaf_prims += count
            for i in range(count):
                seen[order[int(nd["leftOrPrim"]) + i]] += 1
    assert leaf_prims == n
    assert (seen == 1).all()


def test_bvh_degenerate_inputs(oracle_lib):
    """bvh_tests.cpp:165-188."""
    nodes, order = oracle_lib.bvh_build(np.zeros((0, 6), np.float32), 4)
    assert len(nodes) == 0
    nodes, order = oracle_lib.bvh_build(np.array([[0, 0, 0, 1, 1, 1]], np.float32), 4)
    assert len(nodes) == 1 and (int(nodes[0]["packed"]) >> 2) == 1
    same = np.tile(np.array([[1, 2, 3, 1, 2, 3]], np.float32), (100, 1))
    nodes, order = oracle_lib.bvh_build(same, 4)
    assert sum(int(nd["packed"]) >> 2 for nd in nodes) == 100


def _soup_scene(oracle_lib, tris):
    o = oracle_lib.OracleScene(16, 16)
    pos = np.asarray(tris, np.float32).reshape(-1, 3)
    idx = np.arange(pos.shape[0], dtype=np.uint32)
    mesh = o.add_mesh(pos, idx)
    inst = o.add_instance(mesh, None, 0)
    o.commit()
    return o, inst


def test_bvh_traversal_matches_bruteforce(oracle_lib, cases):
    """bvh_tests.cpp:121-163 on the same triangles (seed 7) and rays (seed 123):
    hit/miss agrees, t within 1e-4 relative, and more than 50 hits."""
    o, _ = _soup_scene(oracle_lib, cases["tris7"])
    rays = cases["rays123"]
    bvh = o.trace_rays(rays[:, :3], rays[:, 3:])
    bf, t2, mb = o.trace_bruteforce(rays[:, :3], rays[:, 3:])
    assert np.array_equal(bvh["hit"], bf["hit"])
    h = bf["hit"] == 1
    assert h.sum() > 50
    np.testing.assert_allclose(bvh["t"][h], bf["t"][h], rtol=1e-4)
    # with the same Moeller-Trumbore test the closest triangle is identical
    assert (bvh["prim"][h] == bf["prim"][h]).mean() > 0.999


def test_shadow_rays_agree_with_closest_hit(oracle_lib, cases):
    o, _ = _soup_scene(oracle_lib, cases["tris7"])
    rays = cases["rays123"]
    bvh = o.trace_rays(rays[:, :3], rays[:, 3:])
    occ = o.trace_shadow_rays(rays[:, :3], rays[:, 3:])
    assert np.array_equal(occ, bvh["hit"])


def test_pcg4d_golden(oracle_lib):
    g = np.load(GOLDEN / "pcg4d.npz")
    assert np.array_equal(oracle_lib.pcg4d(g["states"]), g["out"])


def test_env_cdf_golden_and_properties(oracle_lib):
    g = np.load(GOLDEN / "env_cdf.npz")
    cdf, integral = oracle_lib.env_cdf(g["sky"])
    assert np.array_equal(cdf, g["cdf"])
    assert np.float32(integral) == g["integral"]
    h, w = g["sky"].shape[:2]
    rows = cdf[: w * h].reshape(h, w)
    assert (np.diff(rows, axis=1) >= 0).all()
    assert np.allclose(rows[:, -1], 1.0, atol=1e-6)
    marg = cdf[w * h:]
    assert (np.diff(marg) >= 0).all() and abs(marg[-1] - 1.0) < 1e-6
    # integral ~ sum of luminance * sin(theta) * dtheta * dphi
    sky = g["sky"].astype(np.float64)
    lum = 0.2126 * sky[..., 0] + 0.7152 * sky[..., 1] + 0.0722 * sky[..., 2]
    th = (np.arange(h) + 0.5) * np.pi / h
    ref = (lum * np.sin(th)[:, None]).sum() * (np.pi / h) * (2 * np.pi / w)
    assert abs(integral - ref) / ref < 1e-5


def test_readback_and_resolve_semantics(oracle_lib):
    acc = np.array([[2.0, 4.0, 6.0, 2.0], [0.0, 0.0, 0.0, 0.0]], np.float32)
    out = oracle_lib.readback_f32(acc, 2)
    assert np.array_equal(out, np.array([[1, 2, 3, 1], [0, 0, 0, 1]], np.float32))
    out0 = oracle_lib.readback_f32(acc, 0)
    assert (out0[:, :3] == 0).all() and (out0[:, 3] == 1).all()
    rgba8 = oracle_lib.resolve_rgba8(acc, 0.0, 0)
    assert rgba8[0, 3] == 255 and rgba8[0, 0] == 255  # mean 1.0 -> white
    assert (rgba8[1, :3] == 0).all()


def test_tlas_two_instance_leaf_enters_only_the_first(oracle_lib):
    """The reference's TLAS keeps at most one instance per leaf only while
    SAH prefers a split: Bvh.cpp:104 makes a leaf of up to 2 * maxLeafSize
    (= 2 for the TLAS) primitives when no split is cheaper, and its closest-
    hit and shadow walks (intersect.glsl:116-121, 150-152) enter only
    instances[leftOrPrim] of a TLAS leaf. Pinned here on the room scene,
    whose wall box holds the heightfield's box: the reference builder itself
    makes the 2-instance root leaf, the oracle's faithful walk never sees the
    heightfield, and the oracle's all-instance walk agrees with brute force."""
    from miniraytrace_b200 import scenes
    s = scenes.room(48, 27, grid=64)
    boxes = np.stack([np.concatenate([m.positions.min(0), m.positions.max(0)]) for m in s.meshes]).astype(np.float32)
    nodes, order = oracle_lib.bvh_build(boxes, 1)
    assert len(nodes) == 1 and int(nodes[0]["packed"]) >> 2 == 2
    if oracle_lib.load_ref_bvh() is not None:
        r_nodes, r_order = oracle_lib.bvh_build(boxes, 1, use_reference=True)
        assert r_nodes.tobytes() == nodes.tobytes() and np.array_equal(r_order, order)

    o = oracle_lib.OracleScene(48, 27)
    s.apply(o)
    o.commit()
    assert o.unwalked_instances() == 1
    rng = np.random.default_rng(1)
    cam = np.float32(s.camera["position"])
    tg = np.stack([rng.uniform(0, 20, 2000), rng.uniform(0, 4, 2000), rng.uniform(0, 10, 2000)], 1)
    d = (tg - cam) / np.linalg.norm(tg - cam, axis=1, keepdims=True)
    org, d = np.tile(cam, (len(d), 1)), d.astype(np.float32)
    bf, _, mb = o.trace_bruteforce(org, d)
    ok = (bf["hit"] == 1) & (mb >= 1e-5)
    walk = o.trace_rays(org, d)
    # brute force sees both instances; the faithful walk only the walls, so
    # every ray brute force sends into the heightfield comes back with a
    # farther wall hit
    assert len(np.unique(bf["instance"][ok])) == 2
    on_terrain = ok & (bf["t"] < walk["t"] * (1 - 1e-4))
    assert on_terrain.sum() > 300
    assert len(np.unique(bf["instance"][on_terrain])) == 1
    assert len(np.unique(walk["instance"][ok])) == 1
    # shadow rays from just above the floor, up to below the ceiling: only the
    # heightfield (y in [0.05, 0.65]) lies in the way
    p = np.stack([rng.uniform(1, 19, 500), np.full(500, 0.01), rng.uniform(1, 9, 500)], 1).astype(np.float32)
    up = np.tile(np.float32([0, 1, 0]), (500, 1))
    assert (o.trace_shadow_rays(p, up, t_max=1.0) == 0).all()

    o.set_all_leaf_instances(True)
    walk = o.trace_rays(org, d)
    assert np.array_equal(walk["hit"][ok], bf["hit"][ok])
    np.testing.assert_allclose(walk["t"][ok], bf["t"][ok], rtol=1e-4)
    assert (o.trace_shadow_rays(p, up, t_max=1.0) == 1).all()
    o.close()

    b = scenes.box_sphere()
    o = oracle_lib.OracleScene(64, 64)
    b.apply(o)
    o.commit()
    assert o.unwalked_instances() == 0
    o.close()


def test_walk_modes_on_an_instanced_terrain(oracle_lib):
    """The oracle's three ways to find hits, on a small instanced terrain
    (48^2 heightfield, 24 icospheres) whose reference TLAS holds one
    2-instance leaf: the faithful walk differs from brute force in some
    pixels; entering every leaf instance gives brute force's image bit for
    bit; the switches act on render_f32 and render_f64 alike."""
    from miniraytrace_b200 import scenes
    s = scenes.terrain(width=48, height=32, spp=2, grid=48, spheres=24, sky=(64, 32))
    o = oracle_lib.OracleScene(48, 32)
    s.apply(o)
    o.commit()
    assert o.unwalked_instances() == 1
    faithful = o.render_f32(0, 2)
    o.set_all_leaf_instances(True)
    every = o.render_f32(0, 2)
    every64 = o.render_f64(0, 2)
    o.set_all_leaf_instances(False)
    o.set_bruteforce(2)
    brute = o.render_f32(0, 2)
    brute64 = o.render_f64(0, 2)
    o.close()
    assert np.array_equal(every, brute)
    assert np.allclose(every64, brute64, rtol=1e-12, atol=0)
    differ = ~np.all(faithful == brute, axis=-1)
    assert 0 < differ.sum() < 0.02 * differ.size


# ---- pins against the reference's own scene store and env-CDF loop ---------
# (oracle/build_oracle.py compiles core/src/scene/Scene.cpp and the CDF loop
# of core/src/render/Renderer.cpp:620-655 from the reference sources into
# oracle/_ref/; without the reference checkout these tests are skipped.)

def attribute_meshes():
    """Meshes that reach every branch of the reference's attribute code:
    shared vertices, unused vertices (zero normal -> (0, 1, 0)), zero-area
    triangles, degenerate uv triangles (|det| < 1e-12 skipped), tangents
    parallel to the normal (the cross-product fallback), mirrored uvs
    (negative handedness)."""
    from miniraytrace_b200 import scenes
    out = []
    pos, idx, _, _ = scenes.heightfield(48)
    out.append(("heightfield+uv", pos, idx, np.stack([pos[:, 0], pos[:, 2]], 1)))
    ipos, iidx, _ = scenes.icosphere(2)
    out.append(("icosphere", ipos, iidx, None))
    r = np.random.default_rng(8)
    soup = r.uniform(-1, 1, (300, 3)).astype(np.float32)
    sidx = r.integers(0, 280, 600).astype(np.uint32)  # vertices 280..299 unused
    sidx[:30] = np.repeat(sidx[:10], 3)                # zero-area triangles
    uv = r.uniform(0, 1, (300, 2)).astype(np.float32)
    uv[:40] = uv[0]                                    # degenerate uv triangles
    uv[40:80, 0] *= -1                                 # mirrored
    out.append(("soup", soup, sidx, uv))
    flat = np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1], [1, 0, 1]], np.float32)
    fidx = np.array([0, 2, 1, 1, 2, 3], np.uint32)
    fuv = np.array([[0, 0], [0, 0], [0, 1], [0, 1]], np.float32)  # u never changes: tangent fallback
    out.append(("flat", flat, fidx, fuv))
    return out


def engine_attributes(tmp_path, pos, idx, uv):
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    root = Path(__file__).resolve().parents[1]
    host = root / "miniraytrace_b200" / "csrc" / "host"
    exe = tmp_path / "scene_attr_dump"
    if not exe.exists():
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-pthread", "-I", str(host), "-I",
                        str(root / "include"), str(root / "tests" / "host" / "scene_attr_dump.cpp"),
                        str(host / "scene.cpp"), "-o", str(exe)], check=True, capture_output=True)
    pos = np.ascontiguousarray(pos, np.float32)
    idx = np.ascontiguousarray(idx, np.uint32)
    src, dst = tmp_path / "mesh.bin", tmp_path / "attr.bin"
    with open(src, "wb") as f:
        f.write(np.array([pos.shape[0], idx.size, 0 if uv is None else 1], np.uint32).tobytes())
        f.write(pos.tobytes())
        f.write(idx.tobytes())
        if uv is not None:
            f.write(np.ascontiguousarray(uv, np.float32).tobytes())
    subprocess.run([str(exe), str(src), str(dst)], check=True)
    a = np.fromfile(dst, np.float32).reshape(-1, 4)
    nv = pos.shape[0]
    return a[:nv], (a[nv:] if uv is not None else None)


def test_mesh_attributes_equal_the_reference_scene_store(oracle_lib, tmp_path):
    """Normals and tangents: the oracle's restatement and the engine's host
    code (the attributes the GPU reads) equal, bit for bit, what the
    reference's own Scene::addMesh computes (Scene.cpp:13-92)."""
    if oracle_lib.load_ref_scene() is None:
        pytest.skip("reference checkout absent: oracle/_ref/libref_scene.so not built")
    for name, pos, idx, uv in attribute_meshes():
        rn, rt = oracle_lib.ref_mesh_attributes(pos, idx, uv)
        on, ot = oracle_lib.mesh_attributes(pos, idx, uv)
        en, et = engine_attributes(tmp_path, pos, idx, uv)
        assert np.array_equal(on, rn), name
        assert np.array_equal(en[:, :3], rn[:, :3]), name
        if uv is None:
            assert rt is None and ot is None and et is None, name
        else:
            assert np.array_equal(ot, rt), name
            assert np.array_equal(et, rt), name
            if name == "soup":  # mirrored uvs give both handednesses
                assert (rt[:, 3] == -1).any() and (rt[:, 3] == 1).any()


def test_env_cdf_equals_the_reference_loop(oracle_lib):
    """The oracle's CDF (which the device kernel matches bit for bit) equals
    the reference's own loop compiled from Renderer.cpp: conditional rows,
    marginal and integral, on maps with a sun peak, black rows, an all-black
    map (integral clamped to 1e-8), one row, and odd sizes."""
    if oracle_lib.load_ref_envcdf() is None:
        pytest.skip("reference checkout absent: oracle/_ref/libref_envcdf.so not built")
    from miniraytrace_b200 import scenes
    maps = [scenes.procedural_sky(2048, 1024), scenes.procedural_sky(300, 77, sun_sigma_deg=3.0, sun_peak=500.0),
            np.zeros((16, 8, 4), np.float32), scenes.procedural_sky(33, 1)]
    holes = scenes.procedural_sky(128, 64)
    holes[10:20] = 0.0
    maps.append(holes)
    for sky in maps:
        cdf, integral = oracle_lib.env_cdf(sky)
        rcdf, rintegral = oracle_lib.ref_env_cdf(sky)
        assert np.array_equal(cdf, rcdf), sky.shape
        assert np.float32(integral) == np.float32(rintegral), sky.shape


def bvh2_depth(nodes):
    """Levels of a BVH2 (root = 1). The reference's walks (intersect.glsl:
    48-125) pop a node and push both children of an internal one, so a walk
    holds at most `depth` stack entries."""
    left = nodes["leftOrPrim"]
    count = nodes["packed"] >> 2
    best, stack = 0, [(0, 1)]
    while stack:
        n, d = stack.pop()
        best = max(best, d)
        if count[n] == 0:
            stack += [(int(left[n]), d + 1), (int(left[n]) + 1, d + 1)]
    return best


def test_reference_stacks_hold_the_terrain_trees(oracle_lib):
    """The reference walks a BLAS with a fixed 32-entry stack and the TLAS
    with a 16-entry one, without overflow checks (intersect.glsl:51, 96, 132,
    154), while the oracle restating the walks uses 64 entries. On the
    terrain workload the reference builder's trees (4 triangles a BLAS leaf,
    1 instance a TLAS leaf, Renderer.cpp:342-368, 448-508) are shallow enough
    that the reference's stacks never overflow, so the two walks are the
    same: 2,093,058-triangle heightfield and 1,280-triangle icosphere BLASes
    (at most 32 levels), 257-instance TLAS (at most 16). (The largest
    workload's trees, measured once: 19,999,980-triangle heightfield depth
    25; 4,097-instance TLAS depth 16, which fills the reference's TLAS stack
    exactly.)"""
    from miniraytrace_b200 import scenes
    s = scenes.terrain(64, 36, sky=(64, 32))
    bounds = []
    for m in s.meshes:
        a = tri_aabbs(m.positions[m.indices.reshape(-1, 3)])
        depth = bvh2_depth(oracle_lib.bvh_build(a, 4)[0])
        assert depth <= 32, (len(a), depth)
        bounds.append((a[:, :3].min(0), a[:, 3:].max(0)))
    boxes = []
    for mi, xf, _ in s.instances:
        lo, hi = bounds[mi]
        if xf is not None:
            c = np.array([[x, y, z] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])])
            w = c @ xf[:, :3].T.astype(np.float64) + xf[:, 3]
            lo, hi = w.min(0), w.max(0)
        boxes.append(np.concatenate([lo, hi]))
    assert len(boxes) == 257
    depth = bvh2_depth(oracle_lib.bvh_build(np.array(boxes, np.float32), 1)[0])
    assert depth <= 16, depth
