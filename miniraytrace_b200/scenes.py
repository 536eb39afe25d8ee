"""Seeded synthetic scenes for the benchmark configurations.

The reference ships no benchmark scenes (its only HDR asset is missing), so
the configurations are generated here from fixed seeds. A ``SceneSpec`` is a
plain description (numpy arrays + parameters) that ``apply()`` hands to any
object with the scene-building methods of ``miniraytrace_b200.Engine`` -- the
GPU engine or the CPU oracle -- so both see identical inputs.

Configurations:
  box_sphere (C1): open 5-quad box (10 triangles) + UV sphere with 32 slices
      x 16 stacks (992 triangles: a 32-triangle fan at the north pole and 15
      quad bands; the 32 triangles of the last band that touch the south pole
      have zero area), GGX conductor F0 (0.9, 0.6, 0.3), roughness 0.3; sun
      normalize(0.3, 0.8, 0.5), radiance 600, angular radius 0.0465; 256x256,
      16 spp, max bounces 8, firefly clamp off, linear tonemap.
  terrain (C2): 1024x1024-vertex heightfield (2,093,058 triangles) displaced by
      6-octave value-noise fBm (amplitude 0.15, seed 7), 256 instanced
      icospheres (subdivision 3, 1,280 triangles each), per-object materials
      (0.5 diffuse / 0.3 GGX conductor / 0.2 dielectric IOR 1.5), a 2048x1024
      procedural sky (vertical gradient 0.2-1.0 + Gaussian sun of sigma 0.5
      deg, peak 1e4, elevation 30 deg) importance-sampled; 1920x1080, 64 spp,
      max bounces 12.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import abi


@dataclass
class MeshSpec:
    positions: np.ndarray
    indices: np.ndarray
    normals: np.ndarray | None = None
    uvs: np.ndarray | None = None


@dataclass
class SceneSpec:
    name: str
    meshes: list = field(default_factory=list)            # MeshSpec
    materials: list = field(default_factory=list)         # dict of material_desc kwargs
    instances: list = field(default_factory=list)         # (mesh index, xform 3x4 or None, material index or -1)
    lights: list = field(default_factory=list)            # dict of light_desc kwargs
    environment: np.ndarray | None = None                 # (H, W, 4) float32
    env_rotation: float = 0.0
    env_intensity: float = 1.0
    camera: dict = field(default_factory=dict)            # set_camera kwargs
    settings: dict = field(default_factory=dict)          # set_render_settings kwargs
    spp: int = 16
    meta: dict = field(default_factory=dict)

    @property
    def triangle_count(self) -> int:
        return int(sum(self.meshes[m].indices.size // 3 for m, _, _ in self.instances))

    def apply(self, target):
        """Build the scene on `target` (Engine or OracleScene). Returns ids."""
        target.set_render_settings(**self.settings)
        mesh_ids = [target.add_mesh(m.positions, m.indices, m.normals, m.uvs) for m in self.meshes]
        mat_ids = [target.add_material(**m) for m in self.materials]
        inst_ids = [target.add_instance(mesh_ids[mi], xf, mat_ids[ma] if ma >= 0 else 0)
                    for mi, xf, ma in self.instances]
        light_ids = [target.add_light(**l) for l in self.lights]
        if self.environment is not None:
            target.set_environment(self.environment, self.env_rotation, self.env_intensity)
        if self.camera:
            target.set_camera(**self.camera)
        return dict(meshes=mesh_ids, materials=mat_ids, instances=inst_ids, lights=light_ids)


# ---- geometry helpers -------------------------------------------------------------

def quad(p0, p1, p2, p3):
    """Two triangles (p0, p1, p2), (p0, p2, p3)."""
    pos = np.array([p0, p1, p2, p3], np.float32)
    idx = np.array([0, 1, 2, 0, 2, 3], np.uint32)
    return pos, idx


def uv_sphere(slices=32, stacks=16, radius=1.0, center=(0, 0, 0)):
    """Latitude/longitude sphere with slices*(2*stacks - 1) triangles.

    Vertex rows j = 0..stacks (j = 0 is the north pole, j = stacks the south
    pole, each pole row has `slices + 1` coincident vertices). The first band
    is a fan (one triangle per slice); every other band emits two triangles
    per quad, so the 'slices' triangles that touch the south pole have zero
    area. For 32 x 16 this gives 992 triangles.
    """
    verts, nrms = [], []
    for j in range(stacks + 1):
        theta = math.pi * j / stacks
        for i in range(slices + 1):
            phi = 2.0 * math.pi * i / slices
            if j == 0 or j == stacks:  # exact poles
                n = (0.0, 1.0 if j == 0 else -1.0, 0.0)
            else:
                n = (math.sin(theta) * math.cos(phi), math.cos(theta), math.sin(theta) * math.sin(phi))
            nrms.append(n)
            verts.append((center[0] + radius * n[0], center[1] + radius * n[1], center[2] + radius * n[2]))
    idx = []
    row = slices + 1
    for j in range(stacks):
        for i in range(slices):
            a, b = j * row + i, j * row + i + 1
            c, d = (j + 1) * row + i, (j + 1) * row + i + 1
            if j == 0:
                idx += [a, d, c]  # counter-clockwise seen from outside
            else:
                idx += [a, d, c, a, b, d]
    return np.array(verts, np.float32), np.array(idx, np.uint32), np.array(nrms, np.float32)


def icosphere(subdiv=3):
    """Unit icosphere: 20 * 4**subdiv triangles, outward winding, unit normals."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    v = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    pos = np.array(v, np.float32)
    return pos, np.array(f, np.uint32).reshape(-1), pos.copy()


def value_noise_fbm(x, z, octaves=6, seed=7, base_freq=2.0, gain=0.5):
    """Sum of `octaves` bands of seeded value noise (smoothstep-interpolated
    lattice values in [-1, 1]); band k has frequency base_freq * 2**k and
    weight gain**k; the result is normalised to [-1, 1] peak weight."""
    rng = np.random.default_rng(seed)
    out = np.zeros_like(x, dtype=np.float64)
    norm = 0.0
    for k in range(octaves):
        freq = base_freq * (2 ** k)
        n = int(freq) + 2
        lattice = rng.uniform(-1.0, 1.0, size=(n + 1, n + 1))
        fx = (x * 0.5 + 0.5) * freq
        fz = (z * 0.5 + 0.5) * freq
        ix = np.clip(np.floor(fx).astype(np.int64), 0, n - 1)
        iz = np.clip(np.floor(fz).astype(np.int64), 0, n - 1)
        tx = fx - ix
        tz = fz - iz
        sx = tx * tx * (3 - 2 * tx)
        sz = tz * tz * (3 - 2 * tz)
        v00 = lattice[iz, ix]
        v10 = lattice[iz, ix + 1]
        v01 = lattice[iz + 1, ix]
        v11 = lattice[iz + 1, ix + 1]
        band = (v00 * (1 - sx) + v10 * sx) * (1 - sz) + (v01 * (1 - sx) + v11 * sx) * sz
        w = gain ** k
        out += w * band
        norm += w
    return out / norm


def heightfield(n=1024, amplitude=0.15, seed=7, extent=1.0):
    """n x n vertex grid over [-extent, extent]^2 in xz, y = amplitude * fBm;
    2 (n-1)^2 triangles, normals from central differences."""
    lin = np.linspace(-extent, extent, n, dtype=np.float64)
    X, Z = np.meshgrid(lin, lin)
    Y = amplitude * value_noise_fbm(X, Z, seed=seed)
    pos = np.stack([X, Y, Z], -1).reshape(-1, 3).astype(np.float32)
    dy_dx = np.gradient(Y, lin, axis=1)
    dy_dz = np.gradient(Y, lin, axis=0)
    nrm = np.stack([-dy_dx, np.ones_like(Y), -dy_dz], -1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    i = np.arange(n - 1)
    a = (i[:, None] * n + i[None, :]).reshape(-1)  # row-major (z, x)
    b, c, d = a + 1, a + n, a + n + 1
    idx = np.stack([a, c, b, b, c, d], -1).reshape(-1).astype(np.uint32)
    return pos, idx, nrm.reshape(-1, 3).astype(np.float32), Y


def procedural_sky(w=2048, h=1024, sun_elev_deg=30.0, sun_azim_deg=40.0, sun_sigma_deg=0.5, sun_peak=1e4,
                   lo=0.2, hi=1.0):
    """Equirect RGBA32F sky in the reference's mapping (lights.glsl:17-22:
    u -> phi = 2 pi u, v -> theta = pi v, dir = (sin t cos p, cos t, sin t sin p)).
    Above the horizon the radiance falls linearly from `hi` at the horizon to
    `lo` at the zenith (bluish tint), below it is a constant `lo` ground; a
    Gaussian sun lobe (sigma in degrees, peak radiance) sits at the given
    elevation/azimuth. Alpha = 1."""
    u = (np.arange(w) + 0.5) / w
    v = (np.arange(h) + 0.5) / h
    phi = 2 * np.pi * u[None, :]
    theta = np.pi * v[:, None]
    d = np.stack([np.sin(theta) * np.cos(phi), np.cos(theta) * np.ones_like(phi), np.sin(theta) * np.sin(phi)], -1)
    elev = np.arcsin(np.clip(d[..., 1], -1, 1))
    t = np.clip(elev / (np.pi / 2), 0.0, 1.0)
    base = np.where(elev > 0, hi + (lo - hi) * t, lo)
    tint = np.array([0.75, 0.85, 1.0])
    rgb = base[..., None] * tint
    se, sa = np.radians(sun_elev_deg), np.radians(sun_azim_deg)
    sd = np.array([np.cos(se) * np.cos(sa), np.sin(se), np.cos(se) * np.sin(sa)])
    ang = np.arccos(np.clip(d @ sd, -1, 1))
    sig = np.radians(sun_sigma_deg)
    rgb = rgb + sun_peak * np.exp(-0.5 * (ang / sig) ** 2)[..., None] * np.array([1.0, 0.95, 0.85])
    out = np.ones((h, w, 4), np.float32)
    out[..., :3] = rgb
    return out


# ---- configurations -----------------------------------------------------------------

def heightfield_rows(n=4096, rows=2443, amplitude=0.15, seed=7, extent=1.0):
    """The first `rows` vertex rows (in z) of the n x n heightfield of
    heightfield(n, ...): the same grid and fBm, cropped; 2 (n-1)(rows-1)
    triangles."""
    lin = np.linspace(-extent, extent, n, dtype=np.float64)
    X, Z = np.meshgrid(lin, lin[:rows])
    Y = amplitude * value_noise_fbm(X, Z, seed=seed)
    pos = np.stack([X, Y, Z], -1).reshape(-1, 3).astype(np.float32)
    dy_dx = np.gradient(Y, lin, axis=1)
    dy_dz = np.gradient(Y, lin[:rows], axis=0)
    nrm = np.stack([-dy_dx, np.ones_like(Y), -dy_dz], -1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    a = (np.arange(rows - 1)[:, None] * n + np.arange(n - 1)[None, :]).reshape(-1)
    b, c, d = a + 1, a + n, a + n + 1
    idx = np.stack([a, c, b, b, c, d], -1).reshape(-1).astype(np.uint32)
    return pos, idx, nrm.reshape(-1, 3).astype(np.float32), Y


def large(width=3840, height=2160, spp=1024, max_bounces=16, grid=4096, rows=2443, spheres=4096,
          sky=(4096, 2048), seed=7) -> SceneSpec:
    """C5, the largest run: the 4096^2 fBm heightfield cropped to 2 x 4095 x 2442
    = 19,999,980 triangles, 4,096 config-2 icospheres (1,280 triangles each,
    config-2 material mix) on it, a 4096x2048 sky, 3840x2160, depth 16."""
    s = SceneSpec("large")
    pos, idx, nrm, Y = heightfield_rows(grid, rows, 0.15, seed)
    s.meshes.append(MeshSpec(pos, idx, nrm))
    rng = np.random.default_rng(seed + 1000)
    s.materials.append(dict(base_color=tuple(rng.uniform(0.1, 0.9, 3)), roughness=1.0))
    s.instances.append((0, None, 0))
    ipos, iidx, inrm = icosphere(3)
    s.meshes.append(MeshSpec(ipos, iidx, inrm))
    zmax = -1.0 + 2.0 * (rows - 1) / (grid - 1)
    for k in range(spheres):
        x = rng.uniform(-0.95, 0.95)
        z = rng.uniform(-0.95, zmax - 0.05)
        r = rng.uniform(0.02, 0.1)
        gx = int(round((x + 1) / 2 * (grid - 1)))
        gz = min(int(round((z + 1) / 2 * (grid - 1))), rows - 1)
        y = float(Y[gz, gx]) + 0.5 * r
        kind = rng.uniform()
        if kind < 0.5:
            m = dict(base_color=tuple(rng.uniform(0.1, 0.9, 3)), roughness=1.0)
        elif kind < 0.8:
            m = dict(base_color=tuple(rng.uniform(0.5, 1.0, 3)), metallic=1.0, roughness=float(rng.uniform(0.05, 0.8)))
        else:
            m = dict(base_color=(1.0, 1.0, 1.0), transmission=1.0, ior=1.5, roughness=0.05)
        s.materials.append(m)
        xf = np.array([[r, 0, 0, x], [0, r, 0, y], [0, 0, r, z]], np.float32)
        s.instances.append((1, xf, len(s.materials) - 1))
    s.environment = procedural_sky(*sky)
    s.camera = dict(position=(0.0, 0.55, 2.1 + zmax - 1.0), target=(0.0, 0.0, zmax - 1.0), up=(0.0, 1.0, 0.0),
                    fov_y_deg=45.0)
    s.settings = dict(width=width, height=height, max_bounces=max_bounces, spp_limit=1 << 20,
                      firefly_clamp=0.0, tonemap=abi.MRT_TONEMAP_LINEAR, denoise=False)
    s.spp = spp
    s.meta = dict(grid=grid, rows=rows, spheres=spheres, sky=list(sky), seed=seed)
    return s


def room(width=1920, height=1080, spp=64, max_bounces=12, grid=1024, seed=7, sky=(2048, 1024)) -> SceneSpec:
    """C4: a closed 20 x 4 x 10 room (x, y, z) whose only opening is a 2 x 2
    window in the z = 10 wall, facing the config-2 sky (its sun shines in
    through it), with the config-2 heightfield scaled over the floor as
    terrain, so most of the light is indirect. Diffuse walls (0.75) and
    terrain (0.5); area-weighted terrain normals."""
    s = SceneSpec("room")
    x0, x1, y0, y1, z0, z1 = 0.0, 20.0, 0.0, 4.0, 0.0, 10.0
    wx0, wx1, wy0, wy1 = 9.0, 11.0, 1.5, 3.5
    faces = [
        ((x0, y0, z0), (x1, y0, z0), (x1, y0, z1), (x0, y0, z1)),  # floor
        ((x0, y1, z0), (x0, y1, z1), (x1, y1, z1), (x1, y1, z0)),  # ceiling
        ((x0, y0, z0), (x0, y1, z0), (x1, y1, z0), (x1, y0, z0)),  # wall z = 0
        ((x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0)),  # wall x = 0
        ((x1, y0, z0), (x1, y1, z0), (x1, y1, z1), (x1, y0, z1)),  # wall x = 20
        # wall z = 10 around the window
        ((x0, y0, z1), (wx0, y0, z1), (wx0, y1, z1), (x0, y1, z1)),
        ((wx1, y0, z1), (x1, y0, z1), (x1, y1, z1), (wx1, y1, z1)),
        ((wx0, y0, z1), (wx1, y0, z1), (wx1, wy0, z1), (wx0, wy0, z1)),
        ((wx0, wy1, z1), (wx1, wy1, z1), (wx1, y1, z1), (wx0, y1, z1)),
    ]
    pos = np.concatenate([quad(*f)[0] for f in faces])
    idx = np.concatenate([quad(*f)[1] + 4 * k for k, f in enumerate(faces)]).astype(np.uint32)
    s.meshes.append(MeshSpec(pos, idx))
    s.materials.append(dict(base_color=(0.75, 0.75, 0.75), roughness=1.0))
    s.instances.append((0, None, 0))
    hpos, hidx, _, _ = heightfield(grid, 0.15, seed)
    hpos = hpos.astype(np.float64)
    terrain_pos = np.stack([(hpos[:, 0] + 1.0) * 10.0, hpos[:, 1] * 2.0 + 0.35, (hpos[:, 2] + 1.0) * 5.0], 1)
    s.meshes.append(MeshSpec(terrain_pos.astype(np.float32), hidx))
    s.materials.append(dict(base_color=(0.5, 0.5, 0.5), roughness=1.0))
    s.instances.append((1, None, 1))
    s.environment = procedural_sky(*sky)
    s.camera = dict(position=(2.0, 2.6, 1.5), target=(12.0, 1.0, 8.5), up=(0.0, 1.0, 0.0), fov_y_deg=60.0)
    s.settings = dict(width=width, height=height, max_bounces=max_bounces, spp_limit=1 << 20,
                      firefly_clamp=0.0, tonemap=abi.MRT_TONEMAP_LINEAR, denoise=False)
    s.spp = spp
    s.meta = dict(grid=grid, seed=seed, sky=list(sky))
    return s


def batch_jobs(count=16, seed=3, sky=(2048, 1024)) -> list:
    """C3: `count` seeded variants of config 2 for one batched submission:
    triangle counts log-uniform over 10k-2M (heightfield grid sized to the
    count, 32 icospheres), resolution from {256^2, 512^2, 1280x720,
    1920x1080}, 4-64 spp, depth 8-12. One sky is shared by all jobs."""
    rng = np.random.default_rng(seed)
    shared_sky = procedural_sky(*sky)
    resolutions = [(256, 256), (512, 512), (1280, 720), (1920, 1080)]
    jobs = []
    for j in range(count):
        tris = float(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        grid = int(round(np.sqrt(tris / 2.0))) + 1
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        spp = int(rng.integers(4, 65))
        depth = int(rng.integers(8, 13))
        s = terrain(w, h, spp=spp, max_bounces=depth, grid=grid, spheres=32, sky=(8, 4), seed=int(seed * 100 + j))
        s.environment = shared_sky
        s.name = f"batch{j}"
        s.meta.update(job=j, target_triangles=int(tris))
        jobs.append(s)
    return jobs


def box_sphere(width=256, height=256, spp=16, max_bounces=8, firefly_clamp=0.0) -> SceneSpec:
    """C1: open box + GGX conductor UV sphere under a sun (see module doc)."""
    s = SceneSpec("box_sphere")
    # box x in [-1, 1], y in [0, 2], z in [-1, 1], open towards +z (the camera)
    walls = [
        ((-1, 0, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1), (0.8, 0.8, 0.8)),     # floor, normal +y
        ((-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1), (0.8, 0.8, 0.8)),     # ceiling, normal -y
        ((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1), (0.8, 0.8, 0.8)),   # back, normal +z
        ((-1, 0, 1), (-1, 0, -1), (-1, 2, -1), (-1, 2, 1), (0.8, 0.1, 0.1)),   # left, normal +x
        ((1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1), (0.1, 0.8, 0.1)),       # right, normal -x
    ]
    for p0, p1, p2, p3, col in walls:
        pos, idx = quad(p0, p1, p2, p3)
        s.meshes.append(MeshSpec(pos, idx))
        s.materials.append(dict(base_color=col, roughness=1.0, metallic=0.0))
        s.instances.append((len(s.meshes) - 1, None, len(s.materials) - 1))
    pos, idx, nrm = uv_sphere(32, 16, radius=0.5, center=(0.0, 0.5, 0.0))
    s.meshes.append(MeshSpec(pos, idx, nrm))
    s.materials.append(dict(base_color=(0.9, 0.6, 0.3), roughness=0.3, metallic=1.0))
    s.instances.append((len(s.meshes) - 1, None, len(s.materials) - 1))
    d = np.array([0.3, 0.8, 0.5])
    d = d / np.linalg.norm(d)
    s.lights.append(dict(type=abi.MRT_LIGHT_SUN, direction=tuple(d), radiance=(600.0, 600.0, 600.0),
                         angular_radius=0.0465))
    s.camera = dict(position=(0.0, 1.0, 3.6), target=(0.0, 0.9, 0.0), up=(0.0, 1.0, 0.0), fov_y_deg=45.0)
    s.settings = dict(width=width, height=height, max_bounces=max_bounces, spp_limit=1 << 20,
                      firefly_clamp=firefly_clamp, tonemap=abi.MRT_TONEMAP_LINEAR, denoise=False)
    s.spp = spp
    return s


def terrain(width=1920, height=1080, spp=64, max_bounces=12, grid=1024, spheres=256, sky=(2048, 1024),
            seed=7, firefly_clamp=0.0) -> SceneSpec:
    """C2: fBm heightfield + instanced icospheres + procedural sky (module doc)."""
    s = SceneSpec("terrain")
    pos, idx, nrm, Y = heightfield(grid, 0.15, seed)
    s.meshes.append(MeshSpec(pos, idx, nrm))
    rng = np.random.default_rng(seed + 1000)
    s.materials.append(dict(base_color=tuple(rng.uniform(0.1, 0.9, 3)), roughness=1.0))
    s.instances.append((0, None, 0))
    ipos, iidx, inrm = icosphere(3)
    s.meshes.append(MeshSpec(ipos, iidx, inrm))
    lin = np.linspace(-1, 1, grid)
    for k in range(spheres):
        x, z = rng.uniform(-0.9, 0.9, 2)
        r = rng.uniform(0.02, 0.1)
        gx = int(round((x + 1) / 2 * (grid - 1)))
        gz = int(round((z + 1) / 2 * (grid - 1)))
        y = float(Y[gz, gx]) + 0.5 * r
        kind = rng.uniform()
        if kind < 0.5:
            m = dict(base_color=tuple(rng.uniform(0.1, 0.9, 3)), roughness=1.0)
        elif kind < 0.8:
            m = dict(base_color=tuple(rng.uniform(0.5, 1.0, 3)), metallic=1.0, roughness=float(rng.uniform(0.05, 0.8)))
        else:
            m = dict(base_color=(1.0, 1.0, 1.0), transmission=1.0, ior=1.5, roughness=0.05)
        s.materials.append(m)
        xf = np.array([[r, 0, 0, x], [0, r, 0, y], [0, 0, r, z]], np.float32)
        s.instances.append((1, xf, len(s.materials) - 1))
    s.environment = procedural_sky(*sky)
    s.camera = dict(position=(0.0, 0.55, 2.1), target=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), fov_y_deg=45.0)
    s.settings = dict(width=width, height=height, max_bounces=max_bounces, spp_limit=1 << 20,
                      firefly_clamp=firefly_clamp, tonemap=abi.MRT_TONEMAP_LINEAR, denoise=False)
    s.spp = spp
    s.meta = dict(grid=grid, spheres=spheres, sky=list(sky), seed=seed)
    return s
