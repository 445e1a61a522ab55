"""Seeded synthetic workloads with the shapes the benchmark configurations name.

The reference renders OBJ scenes (Sponza, which is not shipped) through its
Scene class (src/Renderer/Scene.cpp:276-380); these generators stand in for
them with procedural geometry of the stated sizes. Geometry is emitted the way
Scene/BVHGeometry feed the reference builder: per-object chunks of at most
65,535 vertices with 16-bit local indices and one Lambert material each
(BVHGeometry::addTriangleList, src/Renderer/BVHGeometry.cpp:46-62;
BVHBuilder::addTriangleList, src/Renderer/BVHBuilder.cpp:265-280).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

TMAX = 100.0
MATERIAL_LAMBERT = 2


@dataclass
class Scene:
    name: str
    positions: np.ndarray          # float32 [V, 3]
    normals: np.ndarray            # float32 [V, 3]
    chunks: np.ndarray             # uint32 [C, 4]: vertex_start, num_vertex, tri_start, num_tri
    local_idx: np.ndarray          # uint32 [T, 3], local to the chunk
    colors: np.ndarray             # float32 [C, 3]
    lights: np.ndarray             # float32 [L, 8]: pos.xyz, radius, color.xyz, sphereRadius
    meta: dict = field(default_factory=dict)

    @property
    def num_tris(self) -> int:
        return int(self.local_idx.shape[0])

    @property
    def num_vertex(self) -> int:
        return int(self.positions.shape[0])

    def tri_records(self) -> np.ndarray:
        """Triangle records (vertexOffset, i0 | i1 << 16, i2 | matId << 16); chunk c
        uses material c + 1 because the reference builder's material 0 is its
        default white (BVHBuilder.h:73)."""
        rec = np.empty((self.num_tris, 3), dtype=np.uint32)
        for c, (v0, nv, t0, nt) in enumerate(self.chunks.tolist()):
            li = self.local_idx[t0:t0 + nt]
            rec[t0:t0 + nt, 0] = v0
            rec[t0:t0 + nt, 1] = li[:, 0] | (li[:, 1] << 16)
            rec[t0:t0 + nt, 2] = li[:, 2] | np.uint32((c + 1) << 16)
        return rec

    def materials_bytes(self) -> bytes:
        """Material records (48 B: uvec4 type_ids, vec4 color, vec4 params;
        primitive_cpp.glsl:67-72), default white first, as the reference packs them."""
        n = len(self.chunks) + 1
        m = np.zeros((n, 12), dtype=np.float32)
        ti = m.view(np.uint32)
        ti[:, 0] = MATERIAL_LAMBERT
        ti[:, 1:4] = 0xFFFFFFFF
        m[0, 4:7] = 1.0
        m[1:, 4:7] = self.colors
        return m.tobytes()

    def packed_lights_bytes(self) -> bytes:
        """PackedLight records (56 B: iparam + 13 floats; primitive_cpp.glsl:113-117;
        packSphereLight, BVHBuilder.cpp:1250-1262)."""
        L = np.zeros((len(self.lights), 14), dtype=np.float32)
        L.view(np.uint32)[:, 0] = 1  # Light_Sphere
        L[:, 1:9] = self.lights
        return L.tobytes()

    def bounds(self):
        return self.positions.min(axis=0), self.positions.max(axis=0)


class _Builder:
    def __init__(self):
        self.pos, self.nrm, self.idx, self.chunks, self.colors = [], [], [], [], []
        self.nv = 0
        self.nt = 0

    def add(self, pos, nrm, idx, color):
        pos = np.asarray(pos, np.float32)
        nrm = np.asarray(nrm, np.float32)
        idx = np.asarray(idx, np.uint32)
        assert pos.shape[0] <= 65535, "a chunk holds at most 65535 vertices (16-bit local indices)"
        self.chunks.append((self.nv, pos.shape[0], self.nt, idx.shape[0]))
        self.pos.append(pos)
        self.nrm.append(nrm)
        self.idx.append(idx)
        self.colors.append(color)
        self.nv += pos.shape[0]
        self.nt += idx.shape[0]

    def scene(self, name, lights, **meta) -> Scene:
        return Scene(name=name, positions=np.concatenate(self.pos), normals=np.concatenate(self.nrm),
                     chunks=np.array(self.chunks, dtype=np.uint32).reshape(-1, 4),
                     local_idx=np.concatenate(self.idx), colors=np.array(self.colors, np.float32).reshape(-1, 3),
                     lights=np.asarray(lights, np.float32).reshape(-1, 8), meta=meta)


def icosphere(subdiv: int):
    """Unit icosphere: 20 * 4**subdiv faces (1,280 at subdiv 3), 642 vertices at subdiv 3."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts, np.float64), np.array(faces, np.uint32)


def _quad(b: _Builder, p0, p1, p2, p3, color):
    p = np.array([p0, p1, p2, p3], np.float64)
    n = np.cross(p[1] - p[0], p[2] - p[0])
    n = n / np.linalg.norm(n)
    b.add(p, np.repeat(n[None], 4, 0), [[0, 1, 2], [0, 2, 3]], color)


def _box(b: _Builder, lo, hi, color):
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    c = [(x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0), (x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)]
    faces = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)]
    pos, nrm, idx = [], [], []
    for f in faces:
        q = np.array([c[i] for i in f], np.float64)
        n = np.cross(q[1] - q[0], q[2] - q[0])
        n /= np.linalg.norm(n)
        base = len(pos)
        pos += list(q)
        nrm += [n] * 4
        idx += [[base, base + 1, base + 2], [base, base + 2, base + 3]]
    b.add(pos, nrm, idx, color)


def _sphere(b: _Builder, center, radius, color, subdiv=3):
    v, f = icosphere(subdiv)
    b.add(np.asarray(center) + radius * v, v, f, color)


def room_scene(seed: int = 1) -> Scene:
    """Config 1: room [0,4]x[0,4]x[0,3] of 5 axis-aligned wall quads (floor and 4
    walls, no ceiling; 10 tris), 2 axis-aligned boxes (24 tris) and one
    icosphere subdivided 3 times (1,280 tris, radius 0.3, centre uniform in the
    room shrunk by 0.3); a point light at the ceiling centre (2, 2, 3), radius 100."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    W, D, H = 4.0, 4.0, 3.0
    _quad(b, (0, 0, 0), (W, 0, 0), (W, D, 0), (0, D, 0), (0.8, 0.8, 0.8))          # floor
    _quad(b, (0, 0, 0), (0, D, 0), (0, D, H), (0, 0, H), (0.8, 0.2, 0.2))          # x = 0
    _quad(b, (W, 0, 0), (W, 0, H), (W, D, H), (W, D, 0), (0.2, 0.8, 0.2))          # x = 4
    _quad(b, (0, D, 0), (W, D, 0), (W, D, H), (0, D, H), (0.8, 0.8, 0.8))          # y = 4
    _quad(b, (0, 0, 0), (0, 0, H), (W, 0, H), (W, 0, 0), (0.8, 0.8, 0.8))          # y = 0
    _box(b, (0.6, 2.2, 0.0), (1.6, 3.2, 1.4), (0.7, 0.7, 0.7))
    _box(b, (2.5, 1.2, 0.0), (3.3, 2.0, 0.8), (0.7, 0.7, 0.7))
    r = 0.3
    centre = rng.uniform((r, r, r), (W - r, D - r, H - r))
    _sphere(b, centre, r, (0.9, 0.9, 0.2))
    lights = [[2.0, 2.0, 3.0, 100.0, 10.0, 10.0, 10.0, 0.1]]
    return b.scene("room", lights, cam_pos=(2.0, 0.2, 1.5), cam_target=(2.0, 4.0, 1.5), sun_dir=(-0.3, 0.2, -1.0),
                   seed=seed)


def heightfield_scene(seed: int = 2, grid: int = 128, n_spheres: int = 53, extent: float = 20.0,
                      n_lights: int = 16, light_radius: float = 6.0) -> Scene:
    """Config 2 (and its 1M-triangle scale-up for config 4): a grid x grid quad
    heightfield over [0, extent]^2 with heights uniform in [0, 2] (2*grid^2
    tris), plus n_spheres icospheres of 1,280 tris (centres uniform in
    extent x extent x 5, radii log-uniform in [0.2, 1.5]); n_lights point lights
    uniform in the same box."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    h = rng.uniform(0.0, 2.0, size=(grid + 1, grid + 1))
    xs = np.linspace(0.0, extent, grid + 1)
    # split the heightfield into row strips of <= 65535 vertices
    rows_per = max(1, 65535 // (grid + 1) - 1)
    r0 = 0
    while r0 < grid:
        r1 = min(grid, r0 + rows_per)
        ys = xs[r0:r1 + 1]
        X, Y = np.meshgrid(xs, ys, indexing="xy")
        Z = h[r0:r1 + 1, :]
        P = np.stack([X, Y, Z], -1).reshape(-1, 3)
        gy, gx = np.gradient(Z, xs[1] - xs[0])
        N = np.stack([-gx, -gy, np.ones_like(Z)], -1).reshape(-1, 3)
        N /= np.linalg.norm(N, axis=1, keepdims=True)
        nx = grid + 1
        ii, jj = np.meshgrid(np.arange(grid), np.arange(r1 - r0), indexing="xy")
        a = (jj * nx + ii).ravel()
        tri = np.concatenate([np.stack([a, a + 1, a + nx + 1], 1), np.stack([a, a + nx + 1, a + nx], 1)])
        b.add(P, N, tri, (0.5, 0.6, 0.4))
        r0 = r1
    centres = rng.uniform((0.0, 0.0, 0.0), (extent, extent, 5.0), size=(n_spheres, 3))
    radii = np.exp(rng.uniform(math.log(0.2), math.log(1.5), size=n_spheres))
    for k in range(n_spheres):
        _sphere(b, centres[k], radii[k], tuple(rng.uniform(0.2, 0.9, 3)))
    lp = rng.uniform((0.0, 0.0, 0.5), (extent, extent, 5.0), size=(n_lights, 3))
    lights = [[*lp[k], light_radius, 4.0, 4.0, 4.0, 0.1] for k in range(n_lights)]
    return b.scene("heightfield", lights, cam_pos=(extent * 0.5, -3.0, 7.0),
                   cam_target=(extent * 0.5, extent * 0.6, 0.0), sun_dir=(-0.4, 0.3, -1.0), seed=seed)


def scaled_heightfield(seed: int, target_tris: int, extent: float = 20.0) -> Scene:
    """The heightfield + icosphere generator at about target_tris triangles, with
    the ~100K scene's split (one third heightfield, two thirds icospheres)."""
    grid = max(4, int(round(math.sqrt(target_tris / 6.0))))
    n_spheres = max(0, int(round((target_tris - 2 * grid * grid) / 1280.0)))
    return heightfield_scene(seed=seed, grid=grid, n_spheres=n_spheres, extent=extent)


def serving_rays(seed: int, n: int, extent: float = 20.0, lights=None) -> np.ndarray:
    """Mixed rays of a serving job over a heightfield scene, one third each:
    primary (from z = 8 looking down, closest hit), shadow (from a point above the
    terrain towards a light, any hit, tmax = the light distance) and probe-update
    (from a point in the probe box, uniform direction, closest hit). Ray records as
    random_rays; flags bit 0 marks the shadow rays."""
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 8), np.float32)
    kind = rng.integers(0, 3, size=n)
    o = np.empty((n, 3))
    d = rng.normal(size=(n, 3))
    tmax = np.full(n, TMAX)
    p = kind == 0
    o[p] = np.column_stack([rng.uniform(0, extent, (p.sum(), 2)), np.full(p.sum(), 8.0)])
    d[p, 2] = -np.abs(d[p, 2]) - 2.0
    s = kind == 1
    o[s] = rng.uniform((0.0, 0.0, 0.0), (extent, extent, 2.5), size=(s.sum(), 3))
    lp = (np.asarray(lights, np.float64)[:, :3] if lights is not None and len(lights)
          else rng.uniform((0, 0, 0.5), (extent, extent, 5.0), size=(16, 3)))
    tgt = lp[rng.integers(0, len(lp), size=s.sum())]
    d[s] = tgt - o[s]
    tmax[s] = np.linalg.norm(d[s], axis=1)
    q = kind == 2
    o[q] = rng.uniform((0.0, 0.0, 0.5), (extent, extent, 5.0), size=(q.sum(), 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 0:3] = o
    r[:, 3] = tmax
    r[:, 4:7] = d
    r.view(np.uint32)[:, 7] = s.astype(np.uint32)
    return r


def random_triangles(seed: int, n: int) -> Scene:
    """Config 3 scenes: n triangles in the unit cube; each has a vertex uniform in
    [0,1]^3 and two edges of length log-uniform in [1e-3, 1e-1] with uniform direction."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    p0 = rng.uniform(0.0, 1.0, size=(n, 3))
    e = rng.normal(size=(n, 2, 3))
    e /= np.linalg.norm(e, axis=2, keepdims=True)
    ln = np.exp(rng.uniform(math.log(1e-3), math.log(1e-1), size=(n, 2, 1)))
    e *= ln
    P = np.stack([p0, p0 + e[:, 0], p0 + e[:, 1]], 1)
    Nf = np.cross(e[:, 0], e[:, 1])
    Nf /= np.maximum(np.linalg.norm(Nf, axis=1, keepdims=True), 1e-30)
    per = 21845
    for s in range(0, n, per):
        k = min(per, n - s)
        pos = P[s:s + k].reshape(-1, 3)
        nrm = np.repeat(Nf[s:s + k], 3, 0)
        idx = np.arange(3 * k, dtype=np.uint32).reshape(-1, 3)
        b.add(pos, nrm, idx, (0.7, 0.7, 0.7))
    return b.scene(f"random{n}", [], seed=seed)


def random_rays(seed: int, n: int, any_fraction: float = 0.5, tmax: float = TMAX) -> np.ndarray:
    """Config 3 rays: origins uniform in [0,1]^3, directions uniform on the sphere;
    a fraction flagged as any-hit (occlusion) rays. Returns the 32-byte ray records
    as a float32 [n, 8] array (flags stored as raw u32 bits in column 7)."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(0.0, 1.0, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmax
    r[:, 4:7] = d
    flags = (rng.uniform(size=n) < any_fraction).astype(np.uint32)
    r.view(np.uint32)[:, 7] = flags
    return r


PASS_DATA_DTYPE = np.dtype([
    ("frameSize", "<u4", 2), ("invFrameSize", "<f4", 2), ("cameraPos", "<f4", 4), ("cameraDir", "<f4", 4),
    ("frustumCorner00", "<f4", 4), ("frustumCorner10", "<f4", 4), ("frustumCorner01", "<f4", 4),
    ("invProjView", "<f4", 16), ("sunDir", "<f4", 4), ("sunColor", "<f4", 4),
    ("sceneMinExtent", "<f4", 4), ("sceneMaxExtent", "<f4", 4), ("lpfResolution", "<u4", 4)])
assert PASS_DATA_DTYPE.itemsize == 240


def pass_data(scene: Scene, width: int, height: int, fov_deg: float = 70.0, lpf_res=(12, 12, 12),
              cam_pos=None, cam_target=None, aabb=None) -> np.ndarray:
    """PassData as RayTracingPass::fillPassResources fills it (raytracingPass.cpp:39-67):
    frustum corners of a pinhole camera (fov 70 degrees), sun direction normalised,
    scene AABB and light-probe resolution. Returns a 240-byte structured record."""
    cam = np.array(cam_pos if cam_pos is not None else scene.meta["cam_pos"], np.float64)
    tgt = np.array(cam_target if cam_target is not None else scene.meta["cam_target"], np.float64)
    f = tgt - cam
    f /= np.linalg.norm(f)
    up = np.array([0.0, 0.0, 1.0])
    r = np.cross(f, up)
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    th = math.tan(math.radians(fov_deg) * 0.5)
    aspect = width / height
    centre = cam + f
    c00 = centre - r * th * aspect - u * th
    c10 = centre + r * th * aspect - u * th
    c01 = centre - r * th * aspect + u * th
    pd = np.zeros(1, PASS_DATA_DTYPE)
    pd["frameSize"] = (width, height)
    pd["invFrameSize"] = (np.float32(1.0) / np.float32(width), np.float32(1.0) / np.float32(height))
    pd["cameraPos"] = (*cam, 0.0)
    pd["cameraDir"] = (*f, 0.0)
    pd["frustumCorner00"] = (*c00, 1.0)
    pd["frustumCorner10"] = (*c10, 1.0)
    pd["frustumCorner01"] = (*c01, 1.0)
    sd = np.array(scene.meta.get("sun_dir", (0.0, 0.0, -1.0)), np.float64)
    sd /= np.linalg.norm(sd)
    pd["sunDir"] = (*sd, 0.0)
    pd["sunColor"] = (1.0, 0.95, 0.9, 0.0)
    lo, hi = aabb if aabb is not None else scene.bounds()
    pd["sceneMinExtent"] = (*lo, 0.0)
    pd["sceneMaxExtent"] = (*hi, 0.0)
    pd["lpfResolution"] = (*lpf_res, 0)
    return pd


def octahedral_dirs(side: int = 16) -> np.ndarray:
    """side x side octahedral directions (cell centres), index j*side + i; float32 [n, 4]."""
    i = (np.arange(side) + 0.5) / side * 2.0 - 1.0
    U, V = np.meshgrid(i, i, indexing="xy")
    x, y = U.ravel(), V.ravel()
    z = 1.0 - np.abs(x) - np.abs(y)
    neg = z < 0
    xo, yo = x.copy(), y.copy()
    x[neg] = (1.0 - np.abs(yo[neg])) * np.sign(xo[neg])
    y[neg] = (1.0 - np.abs(xo[neg])) * np.sign(yo[neg])
    d = np.stack([x, y, z], 1)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    out = np.zeros((side * side, 4), np.float32)
    out[:, :3] = d
    return out


def sh9_basis(dirs: np.ndarray) -> np.ndarray:
    """SH9 basis weights per direction, constants and order of
    LightProbFieldPass::sampleRays (lightProbFieldPass.cpp:186-199); float32 [n, 9]."""
    d = dirs[:, :3].astype(np.float32)
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    w = np.zeros((len(d), 9), np.float32)
    w[:, 0] = np.float32(0.282095)
    w[:, 1] = np.float32(0.488603) * x
    w[:, 2] = np.float32(0.488603) * z
    w[:, 3] = np.float32(0.488603) * y
    w[:, 4] = np.float32(1.092548) * x * z
    w[:, 5] = np.float32(1.092548) * y * z
    w[:, 6] = np.float32(1.092548) * x * y
    w[:, 7] = np.float32(0.315392) * (np.float32(3.0) * z * z - np.float32(1.0))
    w[:, 8] = np.float32(0.546274) * (x * x - y * y)
    return w


def probe_coords(index, res):
    """Probe indices -> (x, y, z) grid coordinates in the 4x4x4-tiled order of
    getLightProbCoord (lightprobHelpers.glsl:33-61); vectorised over numpy arrays."""
    index = np.asarray(index, np.int64)
    trx, try_ = res[0] // 4, res[1] // 4
    tile, inn = index // 64, index % 64
    z = tile // (trx * try_)
    tile = tile % (trx * try_)
    y, x = tile // trx, tile % trx
    return x * 4 + inn % 4, y * 4 + (inn // 4) % 4, z * 4 + (inn // 16) % 4


def probe_positions(aabb_min, aabb_max, res, index) -> np.ndarray:
    """Probe positions, getLightProbPosition (lightprobHelpers.glsl:63-69) in FP32
    with the shader's operation order: min + (max - min) / res * (coord + 0.5)."""
    x, y, z = probe_coords(index, res)
    out = np.empty((len(np.atleast_1d(index)), 3), np.float32)
    for a, c in enumerate((x, y, z)):
        lo, hi = np.float32(aabb_min[a]), np.float32(aabb_max[a])
        step = (hi - lo) / np.float32(res[a])
        out[:, a] = lo + step * (c.astype(np.float32) + np.float32(0.5))
    return out


def sh9_from_images16(sh16, res, probes) -> np.ndarray:
    """The SH9 of `probes` (FP32 [n, 27], coefficient-major: j * 3 + channel) as
    fetchSH9 reads it from the 7 RGBA16F images (lightprob/fetchSH_inline.glsl:6-31,
    layout of storeSH9, storeSH_inline.glsl:6-18)."""
    rx, ry, rz = res
    img = np.asarray(sh16, np.uint16).view(np.float16).astype(np.float32).reshape(7, rz, ry, rx, 4)
    x, y, z = probe_coords(np.asarray(probes), res)
    out = np.zeros((len(x), 27), np.float32)
    out[:, 0:3] = img[0, z, y, x, 0:3]
    for j in range(1, 9):
        for ch in range(3):
            image = 1 + 2 * ch if j <= 4 else 2 + 2 * ch
            comp = j - 1 if j <= 4 else j - 5
            out[:, 3 * j + ch] = img[image, z, y, x, comp]
    return out


def instanced_clusters(seed: int, n_clusters: int = 12, tris_per_cluster: int = 600) -> Scene:
    """A two-level scene for the reference's TLAS/BLAS traversal: n_clusters
    objects, each one chunk (one BLAS instance when built with
    BVHBuilder::addBlas): random triangles (edges log-uniform in [0.1, 0.6])
    in a box of side 1..2.5 placed uniformly in [0, 10]^3, so instances overlap
    now and then; a point light at the centre."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    centres = []
    for c in range(n_clusters):
        side = rng.uniform(1.0, 2.5)
        lo = rng.uniform(0.0, 10.0 - side, size=3)
        centres.append(lo + 0.5 * side)
        n = tris_per_cluster
        p0 = lo + rng.uniform(0.0, side, size=(n, 3))
        e = rng.normal(size=(n, 2, 3))
        e /= np.linalg.norm(e, axis=2, keepdims=True)
        e *= np.exp(rng.uniform(math.log(0.1), math.log(0.6), size=(n, 2, 1)))
        P = np.stack([p0, p0 + e[:, 0], p0 + e[:, 1]], 1)
        Nf = np.cross(e[:, 0], e[:, 1])
        Nf /= np.maximum(np.linalg.norm(Nf, axis=1, keepdims=True), 1e-30)
        b.add(P.reshape(-1, 3), np.repeat(Nf, 3, 0), np.arange(3 * n, dtype=np.uint32).reshape(-1, 3),
              tuple(rng.uniform(0.2, 0.9, 3)))
    return b.scene(f"clusters{n_clusters}", [(5.0, 5.0, 5.0, 20.0, 1.0, 1.0, 1.0, 0.1)], seed=seed,
                   centres=np.array(centres, np.float32))


def occlusion_rays(seed: int, n: int, extent: float = 10.0, targets=None) -> np.ndarray:
    """Any-hit rays for the two-level scene: origins uniform in [0, extent]^3
    (some inside instance boxes), tmax log-uniform in [0.1, 20], directions
    uniform -- or, with `targets`, two rays in three aimed at a random target
    point (an instance centre) with a little jitter; every ray flagged any-hit."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(0.0, extent, size=(n, 3))
    d = rng.normal(size=(n, 3))
    if targets is not None:
        aim = rng.uniform(size=n) < 2.0 / 3.0
        t = np.asarray(targets, np.float64)[rng.integers(len(targets), size=n)]
        d = np.where(aim[:, None], t - o + rng.normal(scale=0.3, size=(n, 3)), d)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = np.exp(rng.uniform(math.log(0.1), math.log(20.0), n))
    r[:, 4:7] = d
    r.view(np.uint32)[:, 7] = 1
    return r
