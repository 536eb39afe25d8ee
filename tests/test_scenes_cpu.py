"""The seeded benchmark scenes have the sizes, windings and value ranges the
configurations call for."""
import numpy as np

from miniraytrace_b200 import scenes


def _areas_and_consistency(pos, idx, nrm):
    t = idx.reshape(-1, 3)
    n = np.cross(pos[t[:, 1]] - pos[t[:, 0]], pos[t[:, 2]] - pos[t[:, 0]])
    area = np.linalg.norm(n, axis=1)
    vn = nrm[t[:, 0]] + nrm[t[:, 1]] + nrm[t[:, 2]]
    return area, (n * vn).sum(1)


def test_uv_sphere_992_triangles_outward():
    pos, idx, nrm = scenes.uv_sphere(32, 16)
    area, d = _areas_and_consistency(pos, idx, nrm)
    assert idx.size // 3 == 992
    assert (area == 0).sum() == 32
    assert (d[area > 0] > 0).all()


def test_icosphere_1280_triangles_outward():
    pos, idx, nrm = scenes.icosphere(3)
    area, d = _areas_and_consistency(pos, idx, nrm)
    assert idx.size // 3 == 1280 and (area > 0).all() and (d > 0).all()
    assert np.allclose(np.linalg.norm(pos, axis=1), 1.0, atol=1e-6)


def test_box_sphere_config():
    s = scenes.box_sphere()
    assert s.triangle_count == 1002
    assert s.settings["width"] == 256 and s.spp == 16 and s.settings["max_bounces"] == 8
    assert s.settings["firefly_clamp"] == 0.0
    d = np.array(s.lights[0]["direction"])
    assert np.allclose(d, np.array([0.3, 0.8, 0.5]) / np.linalg.norm([0.3, 0.8, 0.5]))


def test_heightfield_counts_small():
    pos, idx, nrm, Y = scenes.heightfield(64)
    assert idx.size // 3 == 2 * 63 * 63
    area, d = _areas_and_consistency(pos, idx, nrm)
    assert (area > 0).all() and (d > 0).all()
    assert np.abs(Y).max() <= 0.15 + 1e-9


def test_terrain_config_counts():
    s = scenes.terrain(grid=1024, spheres=256, sky=(64, 32))
    assert s.triangle_count == 2_093_058 + 256 * 1280 == 2_420_738
    assert len(s.instances) == 257
    kinds = [("transmission" in m) for m in s.materials[1:]]
    assert 0.1 < np.mean(kinds) < 0.3


def test_sky_sun_lobe():
    sky = scenes.procedural_sky(2048, 1024)
    assert sky.shape == (1024, 2048, 4) and sky.dtype == np.float32
    assert (sky[..., 3] == 1).all()
    assert 0.9e4 < sky[..., :3].max() < 1.1e4
    assert sky[..., 0].min() >= 0.2 * 0.75 - 1e-6
