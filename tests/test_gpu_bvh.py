"""Device BVH builder: the GPU's LBVH + SAH-optimal collapse must equal the
host reference of the same algorithm byte for byte (nodes and triangle
order), and the engine renders with it (large meshes use it on commit)."""
import numpy as np
import pytest

from miniraytrace_b200 import abi

from test_wide_bvh_cpu import heightfield_mesh, soup_mesh

pytestmark = pytest.mark.gpu


def meshes():
    one = (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]], np.uint32))
    same = (one[0], np.tile(one[1], (50, 1)))
    flat = heightfield_mesh(30, 5)
    flat[0][:, 1] = 0.0
    return {"one": one, "two": soup_mesh(2, 1), "three": soup_mesh(3, 1), "same": same, "flat": flat,
            "soup": soup_mesh(5000, 7), "heightfield": heightfield_mesh(300, 9)}


@pytest.mark.parametrize("name", ["one", "two", "three", "same", "flat", "soup", "heightfield"])
def test_device_lbvh_equals_host(gpu, name):
    pos, idx = meshes()[name]
    e = gpu.Engine(16, 16)
    hn, ho = gpu.build_mesh_bvh(pos, idx, abi.MRTX_BVH_HOST_LBVH)
    dn, do = gpu.build_mesh_bvh(pos, idx, abi.MRTX_BVH_DEVICE_LBVH, engine=e)
    # twice: the builder reuses its scratch
    dn2, do2 = gpu.build_mesh_bvh(pos, idx, abi.MRTX_BVH_DEVICE_LBVH, engine=e)
    e.close()
    assert len(dn) == len(hn)
    assert np.array_equal(do, ho)
    assert dn.tobytes() == hn.tobytes()
    assert dn2.tobytes() == hn.tobytes() and np.array_equal(do2, ho)
