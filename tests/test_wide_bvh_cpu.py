"""The 8-wide compressed BVH (host build through mrtxBuildWideBvh): every
primitive sits in exactly one leaf, every quantised child box contains its
subtree (planes are the exact reals p + q * 2^(e-127), p a multiple of the
scale), nodes are well filled, and a traversal with those boxes reaches the
brute-force closest triangle of every ray."""
import numpy as np
import pytest

import miniraytrace_b200 as mrt


def scale_of(e):
    return np.ldexp(1.0, int(e) - 127)


def grid(node):
    """Per axis: scale and the grid index k of the origin (p = k * s)."""
    s = np.array([scale_of(node["e"][a]) for a in range(3)])
    k = node["p"].astype(np.float64) / s
    assert (k == np.floor(k)).all()
    return s, k


def decode(node, slot):
    # exact in float64 for the grid sizes these tests build
    s, k = grid(node)
    lo = (k + node["qlo"][:, slot]) * s
    hi = (k + node["qhi"][:, slot]) * s
    return lo, hi


def children(node):
    out = []
    internal_rank = 0
    for slot in range(8):
        m = int(node["meta"][slot])
        if m == 0:
            continue
        if (int(node["imask"]) >> slot) & 1:
            out.append((slot, "node", int(node["childBase"]) + internal_rank))
            internal_rank += 1
        else:
            n = bin(m >> 5).count("1")
            off = m & 31
            out.append((slot, "leaf", (int(node["primBase"]) + off, n)))
    return out


def subtree_prims(nodes, order, idx):
    prims = []
    stack = [idx]
    while stack:
        nd = nodes[stack.pop()]
        for slot, kind, ref in children(nd):
            if kind == "node":
                stack.append(ref)
            else:
                prims.extend(order[ref[0]:ref[0] + ref[1]].tolist())
    return prims


def tri_soup(n, seed):
    rng = np.random.default_rng(seed)
    base = rng.uniform(-10, 10, (n, 3))
    tris = np.stack([base, base + rng.uniform(-0.8, 0.8, (n, 3)), base + rng.uniform(-0.8, 0.8, (n, 3))], 1)
    return tris.astype(np.float32)


@pytest.mark.parametrize("leaf", [1, 3])
def test_structure_and_conservative_boxes(mrt_lib, leaf):
    tris = tri_soup(3000, 4)
    boxes = np.concatenate([tris.min(1), tris.max(1)], 1)
    nodes, order = mrt.build_wide_bvh(boxes, leaf)
    assert sorted(order.tolist()) == list(range(len(tris)))
    seen = np.zeros(len(tris), int)
    for ni, nd in enumerate(nodes):
        kids = children(nd)
        assert 1 <= len(kids) <= 8
        for slot, kind, ref in kids:
            lo, hi = decode(nd, slot)
            if kind == "node":
                assert ref < len(nodes)
                prims = subtree_prims(nodes, order, ref)
            else:
                start, n = ref
                assert 1 <= n <= leaf and (int(nd["meta"][slot]) & 31) < 24
                prims = order[start:start + n].tolist()
                seen[prims] += 1
            pb = boxes[prims].astype(np.float64)
            s, k = grid(nd)
            # grid-index comparison: exact for any float coordinates
            assert (k + nd["qlo"][:, slot] <= pb[:, :3] / s).all(), (ni, slot)
            assert (k + nd["qhi"][:, slot] >= pb[:, 3:] / s).all(), (ni, slot)
    assert (seen == 1).all()
    # the SAH collapse fills nodes: well above the two or three children a
    # collapse that only opens oversized subtrees leaves
    fill = np.mean([len(children(nd)) for nd in nodes])
    assert fill > 5.0, fill


def moller_trumbore(o, d, tri):
    e1, e2 = tri[1] - tri[0], tri[2] - tri[0]
    p = np.cross(d, e2)
    det = e1 @ p
    if abs(det) < 1e-12:
        return None
    inv = 1.0 / det
    s = o - tri[0]
    u = (s @ p) * inv
    if u < 0 or u > 1:
        return None
    q = np.cross(s, e1)
    v = (d @ q) * inv
    if v < 0 or u + v > 1:
        return None
    t = (e2 @ q) * inv
    return t if t > 1e-4 else None


def test_traversal_reaches_closest_hit(mrt_lib):
    tris = tri_soup(600, 9).astype(np.float64)
    boxes = np.concatenate([tris.min(1), tris.max(1)], 1).astype(np.float32)
    nodes, order = mrt.build_wide_bvh(boxes, 3)
    rng = np.random.default_rng(3)
    checked = 0
    for _ in range(150):
        o = rng.uniform(-12, 12, 3)
        target = tris[rng.integers(len(tris))].mean(0) + rng.normal(scale=0.2, size=3)
        d = target - o
        d /= np.linalg.norm(d)
        best, best_t = None, np.inf
        for i, tri in enumerate(tris):
            t = moller_trumbore(o, d, tri)
            if t is not None and t < best_t:
                best, best_t = i, t
        if best is None:
            continue
        # walk every node whose decoded box the ray enters before best_t
        inv = 1.0 / np.where(d == 0, 1e-30, d)
        reached = set()
        stack = [0]
        while stack:
            nd = nodes[stack.pop()]
            for slot, kind, ref in children(nd):
                lo, hi = decode(nd, slot)
                t0, t1 = (lo - o) * inv, (hi - o) * inv
                te = max(np.minimum(t0, t1).max(), 0.0)
                tx = min(np.maximum(t0, t1).min(), best_t * (1 + 1e-6))
                if te > tx:
                    continue
                if kind == "node":
                    stack.append(ref)
                else:
                    reached.update(order[ref[0]:ref[0] + ref[1]].tolist())
        assert best in reached
        checked += 1
    assert checked > 40


def test_degenerate_inputs(mrt_lib):
    nodes, order = mrt.build_wide_bvh(np.zeros((0, 6), np.float32))
    assert len(nodes) == 0
    nodes, order = mrt.build_wide_bvh(np.array([[0, 0, 0, 1, 1, 1]], np.float32))
    assert len(nodes) == 1 and list(order) == [0]
    same = np.tile(np.array([[1, 2, 3, 1, 2, 3]], np.float32), (100, 1))
    nodes, order = mrt.build_wide_bvh(same)
    assert sorted(order.tolist()) == list(range(100))
    # flat boxes (a heightfield seen from above has no thickness in leaves)
    flat = np.array([[i, 0, j, i + 1, 0, j + 1] for i in range(10) for j in range(10)], np.float32)
    nodes, order = mrt.build_wide_bvh(flat)
    assert sorted(order.tolist()) == list(range(100))


def soup_mesh(n, seed):
    tris = tri_soup(n, seed)
    return tris.reshape(-1, 3), np.arange(3 * n, dtype=np.uint32).reshape(-1, 3)


def heightfield_mesh(k, seed):
    rng = np.random.default_rng(seed)
    x, z = np.meshgrid(np.linspace(-1, 1, k), np.linspace(-1, 1, k))
    y = 0.05 * rng.standard_normal((k, k))
    pos = np.stack([x, y, z], -1).reshape(-1, 3).astype(np.float32)
    a = (np.arange(k - 1)[:, None] * k + np.arange(k - 1)[None, :]).ravel()
    idx = np.concatenate([np.stack([a, a + 1, a + k], 1), np.stack([a + 1, a + k + 1, a + k], 1)])
    return pos, idx.astype(np.uint32)


@pytest.mark.parametrize("builder", [0, 1])
def test_mesh_builders_structure(mrt_lib, builder):
    pos, idx = soup_mesh(2000, 11)
    tris = pos[idx]
    boxes = np.concatenate([tris.min(1), tris.max(1)], 1)
    nodes, order = mrt.build_mesh_bvh(pos, idx, builder)
    assert sorted(order.tolist()) == list(range(len(idx)))
    for ni, nd in enumerate(nodes):
        s, k = grid(nd)
        for slot, kind, ref in children(nd):
            prims = subtree_prims(nodes, order, ref) if kind == "node" else order[ref[0]:ref[0] + ref[1]].tolist()
            pb = boxes[prims].astype(np.float64)
            assert (k + nd["qlo"][:, slot] <= pb[:, :3] / s).all(), (ni, slot)
            assert (k + nd["qhi"][:, slot] >= pb[:, 3:] / s).all(), (ni, slot)


def test_layout_follows_subtree_sizes(mrt_lib):
    """The depth-first layout the device emission reproduces level by level:
    a node's internal children are consecutive from childBase; child r's own
    children start after all children of its parent plus the subtrees of
    children 0..r-1; its primitives start after the parent's leaf primitives
    plus the primitives of children 0..r-1."""
    for builder, (pos, idx) in [(0, soup_mesh(1500, 2)), (1, soup_mesh(1500, 2)), (1, heightfield_mesh(40, 3))]:
        nodes, order = mrt.build_mesh_bvh(pos, idx, builder)
        below, prims = {}, {}

        def sizes(w):
            nb, npr = 0, 0
            for slot, kind, ref in children(nodes[w]):
                if kind == "node":
                    b, p = sizes(ref)
                    nb += 1 + b
                    npr += p
                else:
                    npr += ref[1]
            below[w], prims[w] = nb, npr
            return nb, npr

        sizes(0)
        assert 1 + below[0] == len(nodes) and prims[0] == len(idx)
        for w, nd in enumerate(nodes):
            kids = children(nd)
            internal = [ref for _, kind, ref in kids if kind == "node"]
            leaf_prims = sum(ref[1] for _, kind, ref in kids if kind == "leaf")
            assert internal == list(range(int(nd["childBase"]), int(nd["childBase"]) + len(internal)))
            next_child = int(nd["childBase"]) + len(internal)
            next_prim = int(nd["primBase"]) + leaf_prims
            for c in internal:
                assert int(nodes[c]["childBase"]) == next_child and int(nodes[c]["primBase"]) == next_prim, (w, c)
                next_child += below[c]
                next_prim += prims[c]


def test_lbvh_degenerate_and_tiny_meshes(mrt_lib):
    one = (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]], np.uint32))
    same = (np.tile(one[0], (1, 1)), np.tile(one[1], (50, 1)))  # 50 identical triangles
    flat = heightfield_mesh(12, 1)
    flat[0][:, 1] = 0.0
    for pos, idx in (one, same, flat, soup_mesh(2, 1), soup_mesh(3, 1)):
        nodes, order = mrt.build_mesh_bvh(pos, idx, 1)
        assert sorted(order.tolist()) == list(range(len(idx)))
        assert 1 <= len(nodes) <= max(1, len(idx))


def test_mesh_builder_rejects_bad_input(mrt_lib):
    pos, idx = soup_mesh(10, 1)
    with pytest.raises(mrt.MrtError):
        mrt.build_mesh_bvh(pos, idx + 100, 1)
    with pytest.raises(mrt.MrtError):
        mrt.build_mesh_bvh(pos, idx, 2)  # device builder without an engine


def test_instance_tree_has_one_instance_per_leaf():
    """The engine's TLAS (binary build with leaf size 1, collapsed with one
    primitive per leaf) puts every instance in a leaf of its own, even for
    nested and coincident boxes, where the reference's build makes
    2-instance leaves (Bvh.cpp:104) whose second instance its traversal
    never enters (intersect.glsl:116-121): the room's wall box holding the
    heightfield's, and a random set of nested, overlapping and equal boxes."""
    from miniraytrace_b200 import scenes
    s = scenes.room(48, 27, grid=64)
    room = np.stack([np.concatenate([m.positions.min(0), m.positions.max(0)]) for m in s.meshes])
    rng = np.random.default_rng(11)
    c = rng.uniform(-5, 5, (300, 3))
    r = rng.exponential(1.0, (300, 1)) * rng.uniform(0.2, 1.0, (300, 3))
    boxes = np.concatenate([c - r, c + r], 1)
    boxes[100:120] = boxes[0]                  # equal boxes
    boxes[120:140, :3] = boxes[0, :3] - 1.0    # boxes holding box 0
    boxes[120:140, 3:] = boxes[0, 3:] + 1.0
    for b in (room, boxes):
        nodes, order = mrt.build_wide_bvh(b.astype(np.float32), max_leaf_prims=1)
        per_leaf = [ref[1] for nd in nodes for _, kind, ref in children(nd) if kind == "leaf"]
        assert per_leaf and all(n == 1 for n in per_leaf)
        assert sorted(subtree_prims(nodes, order, 0)) == list(range(len(b)))


def boxes_as_triangles(boxes):
    """The engine's input to the device builder for an instance tree: each
    box (lo, hi) becomes the degenerate triangle (lo, hi, lo)."""
    b = np.asarray(boxes, np.float32)
    pos = np.empty((2 * len(b), 3), np.float32)
    pos[0::2], pos[1::2] = b[:, :3], b[:, 3:]
    k = np.arange(len(b), dtype=np.uint32)
    return pos, np.stack([2 * k, 2 * k + 1, 2 * k], 1)


def test_instance_boxes_through_the_mesh_builder():
    """The TLAS the device builds (mrtxSetBvhBuildThresholds): instance boxes
    fed to the mesh builder as degenerate triangles. Checked here on its host
    reference (the LBVH the device build equals node for node): every
    triangle's box is exactly its instance's box, every instance sits in a
    leaf of its own, also for nested and equal boxes, and every quantised
    child box holds the instance boxes below it."""
    rng = np.random.default_rng(5)
    c = rng.uniform(-5, 5, (2500, 3))
    r = rng.exponential(1.0, (2500, 1)) * rng.uniform(0.2, 1.0, (2500, 3))
    boxes = np.concatenate([c - r, c + r], 1).astype(np.float32)
    boxes[100:120] = boxes[0]
    boxes[120:140, :3] = boxes[0, :3] - 1.0
    boxes[120:140, 3:] = boxes[0, 3:] + 1.0
    for b in (boxes[:1], boxes[:2], boxes[:3], boxes):
        pos, idx = boxes_as_triangles(b)
        tri = pos[idx]
        assert np.array_equal(np.concatenate([tri.min(1), tri.max(1)], 1), b)
        nodes, order = mrt.build_mesh_bvh(pos, idx, builder=1, max_leaf_prims=1)
        assert sorted(order.tolist()) == list(range(len(b)))
        per_leaf = [ref[1] for nd in nodes for _, kind, ref in children(nd) if kind == "leaf"]
        assert per_leaf and all(n == 1 for n in per_leaf)
        assert sorted(subtree_prims(nodes, order, 0)) == list(range(len(b)))
        for ni, nd in enumerate(nodes):
            s, k = grid(nd)
            for slot, kind, ref in children(nd):
                prims = subtree_prims(nodes, order, ref) if kind == "node" else order[ref[0]:ref[0] + ref[1]].tolist()
                pb = b[prims].astype(np.float64)
                assert (k + nd["qlo"][:, slot] <= pb[:, :3] / s).all(), (ni, slot)
                assert (k + nd["qhi"][:, slot] >= pb[:, 3:] / s).all(), (ni, slot)


def test_host_builder_trees_are_unchanged():
    """The host's binned-SAH builder and the 8-wide collapse, pinned by a
    hash of their output on seeded inputs (boxes with nested and equal
    members, a triangle soup, a heightfield): a change of the host trees,
    which the measured traversal costs were taken with, shows up here."""
    import hashlib

    def boxes(n, seed):
        rng = np.random.default_rng(seed)
        c = rng.uniform(-5, 5, (n, 3))
        r = rng.exponential(1.0, (n, 1)) * rng.uniform(0.2, 1.0, (n, 3))
        b = np.concatenate([c - r, c + r], 1).astype(np.float32)
        if n > 40:
            b[10:20] = b[0]
            b[20:30, :3] = b[0, :3] - 1
            b[20:30, 3:] = b[0, 3:] + 1
        return b

    def digest(nodes, order):
        return hashlib.sha256(nodes.tobytes() + order.tobytes()).hexdigest()[:16]

    expected = {
        "boxes1_leaf1": "c1d5f41ce809fa25", "boxes1_leaf3": "c1d5f41ce809fa25",
        "boxes2_leaf1": "69fd58385c8c5ec6", "boxes2_leaf3": "df927126a9dfd8b7",
        "boxes3_leaf1": "ece8ff83899983f7", "boxes3_leaf3": "0d92900593e276ae",
        "boxes7_leaf1": "3d63154ff7b29788", "boxes7_leaf3": "3d63154ff7b29788",
        "boxes100_leaf1": "8cb71f891b5ecf8c", "boxes100_leaf3": "062ce40d7f642c5f",
        "boxes1000_leaf1": "a61b148f69d79feb", "boxes1000_leaf3": "0e7ed9077243481d",
        "boxes5000_leaf1": "2b0c017692ffb5b4", "boxes5000_leaf3": "930b0d8062c56333",
        "soup3000": "ff09c97e70e2a48a", "hf40": "f8bea9d16356041f",
    }
    got = {}
    for n in (1, 2, 3, 7, 100, 1000, 5000):
        for leaf in (1, 3):
            got[f"boxes{n}_leaf{leaf}"] = digest(*mrt.build_wide_bvh(boxes(n, n), leaf))
    for name, (p, i) in {"soup3000": soup_mesh(3000, 4), "hf40": heightfield_mesh(40, 3)}.items():
        got[name] = digest(*mrt.build_mesh_bvh(p, i, 0))
    assert got == expected
