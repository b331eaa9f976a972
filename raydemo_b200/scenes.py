"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference ships no benchmark scenes for these configurations, so every
scene here is procedural and fully determined by its seed.
"""
from __future__ import annotations

import numpy as np

# ---------------------------------------------------------------- microbench


def random_triangles(n_tris: int, seed: int = 0, mean_edge: float = 0.005, sigma: float = 0.5) -> np.ndarray:
    """`n_tris` random triangles, returned as float32 vertex positions (n, 3, 3).

    Centroids are uniform in the unit cube; each vertex sits at the centroid
    plus an isotropic unit direction times a lognormal(ln mean_edge, sigma)
    length, which gives random orientations and lognormal edge lengths.
    """
    rng = np.random.default_rng(seed)
    c = rng.random((n_tris, 1, 3))
    g = rng.standard_normal((n_tris, 3, 3))
    g /= np.linalg.norm(g, axis=2, keepdims=True)
    length = rng.lognormal(np.log(mean_edge), sigma, (n_tris, 3, 1))
    return (c + g * length).astype(np.float32)


def incoherent_rays(n_rays: int, seed: int = 1, tmax: float = 1e30) -> np.ndarray:
    """Rays as (n, 8) float32: origin uniform in the unit cube, direction
    uniform on the sphere; columns are ox, oy, oz, tmax, dx, dy, dz, 0."""
    rng = np.random.default_rng(seed)
    o = rng.random((n_rays, 3))
    d = rng.standard_normal((n_rays, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n_rays, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmax
    r[:, 4:7] = d
    return r


def coherent_rays(w: int = 2048, h: int = 2048, origin=(0.5, 0.5, -1.5), fov_deg: float = 45.0, tmax: float = 1e30) -> np.ndarray:
    """One pinhole ray per pixel centre, looking along +z at the unit cube."""
    o = np.asarray(origin, np.float64)
    k = np.tan(np.radians(fov_deg) * 0.5)
    xs = ((np.arange(w) + 0.5) / w * 2.0 - 1.0) * k * (w / h)
    ys = (1.0 - (np.arange(h) + 0.5) / h * 2.0) * k
    X, Y = np.meshgrid(xs, ys)
    d = np.stack([X, Y, np.ones_like(X)], axis=-1).reshape(-1, 3)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((w * h, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmax
    r[:, 4:7] = d
    return r


def triangle_soup_mesh(tris: np.ndarray):
    """Vertex attributes (PxyzNxyzTuv, 8 floats per vertex) and indices for a
    triangle soup, as the scene API takes them."""
    n = len(tris)
    attrs = np.zeros((n * 3, 8), np.float32)
    attrs[:, 0:3] = tris.reshape(-1, 3)
    attrs[:, 5] = 1.0
    idx = np.arange(n * 3, dtype=np.uint32)
    return attrs, idx


def tri_aabbs(tris: np.ndarray) -> np.ndarray:
    return np.concatenate([tris.min(axis=1), tris.max(axis=1)], axis=1).astype(np.float32)


# ---------------------------------------------------------------- render scenes
#
# A scene spec is a plain dict that both this library's API and the reference
# build from the same calls, in the same order (so every index matches):
#   textures:  [(rgba (h, w, 4) uint8, is_srgb, generate_mipmaps)]
#   materials: [dict of AddMaterial keyword arguments]
#   meshes:    [(attrs (n, stride) float32, indices uint32, shapes [(mat, back_mat, start, count)], layout)]
#   instances: [(mesh, xform (16,) float32 column-major)]
#   lights:    [dict of AddLight keyword arguments]
#   env:       dict of SetEnvironment keyword arguments
#   camera:    dict of camera_desc_t fields
# Texture indices count from 2: the scene's first two textures are its default
# environment and normal maps.

def icosphere(subdiv: int, radius: float = 1.0):
    """Icosahedron subdivided `subdiv` times (20 * 4^subdiv triangles),
    projected to the sphere. Returns (positions (v, 3), indices (t, 3))."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1),
         (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
         (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
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
    return (np.array(verts) * radius).astype(np.float32), np.array(faces, np.uint32)


def _quad(p0, p1, p2, p3, n):
    """Two triangles (p0 p1 p2, p0 p2 p3) as PxyzNxyzTuv rows."""
    uv = [(0, 0), (1, 0), (1, 1), (0, 1)]
    rows = [list(p) + list(n) + list(t) for p, t in zip((p0, p1, p2, p3), uv)]
    return np.array(rows, np.float32), np.array([0, 1, 2, 0, 2, 3], np.uint32)


def _box(size, yaw, center):
    """12-triangle box (flat normals) of the given size, rotated by yaw about y."""
    sx, sy, sz = (s / 2.0 for s in size)
    c, s = np.cos(yaw), np.sin(yaw)
    R = np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    faces = [((1, 0, 0), [(1, -1, -1), (1, 1, -1), (1, 1, 1), (1, -1, 1)]), ((-1, 0, 0), [(-1, -1, 1), (-1, 1, 1), (-1, 1, -1), (-1, -1, -1)]),
             ((0, 1, 0), [(-1, 1, -1), (-1, 1, 1), (1, 1, 1), (1, 1, -1)]), ((0, -1, 0), [(-1, -1, 1), (-1, -1, -1), (1, -1, -1), (1, -1, 1)]),
             ((0, 0, 1), [(1, -1, 1), (1, 1, 1), (-1, 1, 1), (-1, -1, 1)]), ((0, 0, -1), [(-1, -1, -1), (-1, 1, -1), (1, 1, -1), (1, -1, -1)])]
    rows, idx = [], []
    for n, corners in faces:
        pts = [R @ np.array([cx * sx, cy * sy, cz * sz]) + np.array(center) for cx, cy, cz in corners]
        a, i = _quad(*pts, R @ np.array(n, np.float64))
        idx.append(i + 4 * len(rows))
        rows.append(a)
    return np.concatenate(rows), np.concatenate(idx)


def _concat(parts):
    """[(attrs, idx, material)] -> one mesh with one two-sided shape per part."""
    attrs, idx, shapes, base = [], [], [], 0
    for a, i, m in parts:
        shapes.append((m, m, sum(len(x) for x in idx), len(i)))
        idx.append(i + base)
        attrs.append(a)
        base += len(a)
    return np.concatenate(attrs).astype(np.float32), np.concatenate(idx).astype(np.uint32), shapes


def cornell_box(seed: int = 0, w: int = 256, h: int = 256, max_bounces: int = 4) -> dict:
    """The small render configuration: a Cornell-style box from `seed` --
    five axis-aligned wall quads (10 triangles), two boxes (24 triangles)
    rotated U[0, 45 deg] about y, an icosphere of subdivision 3 (1,280
    triangles, radius 0.2) and a 0.3 x 0.3 quad light of strength 15 (2
    triangles); 1,316 triangles in all. Lambertian materials (Oren-Nayar with roughness 0) with
    albedo U[0.2, 0.8] per channel."""
    rng = np.random.default_rng(seed)
    white = np.full((1, 1, 4), 255, np.uint8)
    spec = {"textures": [(white, False, False)], "materials": [], "meshes": [], "instances": [], "lights": [],
            "env": {"env_col": (0.0, 0.0, 0.0)}}
    tex = 2

    def diffuse():
        spec["materials"].append({"type": 0, "main_color": tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)), "main_texture": tex,
                                  "roughness": 0.0})
        return len(spec["materials"]) - 1

    parts = []
    walls = [((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1), (0, 1, 0)), ((0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0), (0, -1, 0)),
             ((0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1), (0, 0, -1)), ((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0), (1, 0, 0)),
             ((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1), (-1, 0, 0))]
    for p0, p1, p2, p3, n in walls:
        a, i = _quad(p0, p1, p2, p3, n)
        parts.append((a, i, diffuse()))
    for size, center in (((0.25, 0.5, 0.25), (0.68, 0.25, 0.68)), ((0.25, 0.25, 0.25), (0.3, 0.125, 0.35))):
        yaw = np.deg2rad(rng.uniform(0.0, 45.0))
        a, i = _box(size, yaw, center)
        parts.append((a, i, diffuse()))
    spec["materials"].append({"type": 3, "main_color": (1.0, 1.0, 1.0), "main_texture": tex, "strength": 15.0})
    light = len(spec["materials"]) - 1
    a, i = _quad((0.35, 0.999, 0.35), (0.35, 0.999, 0.65), (0.65, 0.999, 0.65), (0.65, 0.999, 0.35), (0, -1, 0))
    parts.append((a, i, light))
    attrs, idx, shapes = _concat(parts)
    spec["meshes"].append((attrs, idx, shapes, 0))
    spec["instances"].append((0, np.eye(4, dtype=np.float32).reshape(-1)))
    # the icosphere: its own mesh, placed by its instance transform
    pos, faces = icosphere(3, 0.2)
    nrm = pos / np.linalg.norm(pos, axis=1, keepdims=True)
    uv = np.stack([0.5 + np.arctan2(nrm[:, 2], nrm[:, 0]) / (2 * np.pi), 0.5 - np.arcsin(nrm[:, 1]) / np.pi], axis=1)
    sphere_mat = diffuse()
    sattrs = np.concatenate([pos, nrm, uv], axis=1).astype(np.float32)
    spec["meshes"].append((sattrs, faces.reshape(-1), [(sphere_mat, sphere_mat, 0, faces.size)], 0))
    xf = np.eye(4, dtype=np.float32)
    xf[3, 0:3] = (0.62, 0.7, 0.3)  # floating in front of the tall box
    spec["instances"].append((1, xf.reshape(-1)))
    spec["camera"] = {"type": 0, "filter": 1, "dtype": 0, "origin": (0.5, 0.5, -1.0), "fwd": (0.0, 0.0, 1.0), "up": (0.0, 1.0, 0.0),
                      "fov": 45.0, "gamma": 1.0, "max_total_depth": max_bounces, "max_diff_depth": max_bounces,
                      "termination_start_depth": max_bounces}
    spec["size"] = (w, h)
    return spec


def lightmap_box(seed: int = 0, res: int = 128, max_bounces: int = 4, overlap: bool = False) -> dict:
    """The Cornell box of `seed` baked to a lightmap: a Geo camera on the room
    instance (walls, boxes and light, 18 quads) whose second UV layer packs
    each quad into its own cell of a 5 x 4 atlas over a res x res framebuffer
    (5 % margins, so texels between cells stay uncovered and show the
    background). overlap: the two boxes' twelve faces share one cell (the
    first triangle in mesh order takes each texel). The environment is a dim
    grey, the paths up to max_bounces long."""
    spec = cornell_box(seed, res, res, max_bounces)
    attrs, idx, shapes, _ = spec["meshes"][0]
    n_quads = len(attrs) // 4
    uv1 = np.zeros((len(attrs), 2), np.float32)
    m = 0.05
    for q in range(n_quads):
        cell = 5 if overlap and 5 <= q < 17 else q
        col, row = cell % 5, cell // 5
        for k in range(4):
            u, v = attrs[4 * q + k, 6:8]
            uv1[4 * q + k] = ((col + m + u * (1 - 2 * m)) / 5.0, (row + m + v * (1 - 2 * m)) / 4.0)
    spec["meshes"][0] = (np.concatenate([attrs, uv1], axis=1).astype(np.float32), idx, shapes, 1)
    spec["env"] = {"env_col": (0.1, 0.1, 0.1)}
    spec["camera"] = {"type": 2, "mi_index": 0, "uv_index": 1, "gamma": 1.0, "max_total_depth": max_bounces,
                      "max_diff_depth": max_bounces, "termination_start_depth": max_bounces}
    return spec


def spec_triangles(spec: dict) -> int:
    return int(sum(len(m[1]) // 3 for m in spec["meshes"]))


# ---------------------------------------------------------------- batched form

_ICO_V = np.array([(-1, 1.618033988749895, 0), (1, 1.618033988749895, 0), (-1, -1.618033988749895, 0), (1, -1.618033988749895, 0),
                   (0, -1, 1.618033988749895), (0, 1, 1.618033988749895), (0, -1, -1.618033988749895), (0, 1, -1.618033988749895),
                   (1.618033988749895, 0, -1), (1.618033988749895, 0, 1), (-1.618033988749895, 0, -1), (-1.618033988749895, 0, 1)])
_ICO_F = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
                   (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)])


def grid_sphere(level: int):
    """Icosphere with 20 * 4^level triangles: each icosahedron face split into
    an n x n triangle grid (n = 2^level) and projected to the unit sphere.
    Vertices on shared edges are repeated per face. Returns (positions (v, 3)
    float64, indices (t, 3) uint32)."""
    n = 1 << level
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    keep = ii + jj <= n
    I, J = ii[keep], jj[keep]                       # barycentric grid of one face
    vid = -np.ones((n + 1, n + 1), np.int64)
    vid[I, J] = np.arange(len(I))
    a, b = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    up = a + b <= n - 1
    t_up = np.stack([vid[a[up], b[up]], vid[a[up] + 1, b[up]], vid[a[up], b[up] + 1]], 1)
    dn = a + b <= n - 2
    t_dn = np.stack([vid[a[dn] + 1, b[dn]], vid[a[dn] + 1, b[dn] + 1], vid[a[dn], b[dn] + 1]], 1)
    tri1 = np.concatenate([t_up, t_dn])
    V = _ICO_V / np.linalg.norm(_ICO_V, axis=1, keepdims=True)
    p0, p1, p2 = V[_ICO_F[:, 0]], V[_ICO_F[:, 1]], V[_ICO_F[:, 2]]
    w1, w2 = I / n, J / n
    pts = p0[:, None, :] + (p1 - p0)[:, None, :] * w1[None, :, None] + (p2 - p0)[:, None, :] * w2[None, :, None]
    pts = pts.reshape(-1, 3)
    pts /= np.linalg.norm(pts, axis=1, keepdims=True)
    faces = (tri1[None, :, :] + (np.arange(20) * len(I))[:, None, None]).reshape(-1, 3)
    return pts, faces.astype(np.uint32)


def value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """3D value noise in [-1, 1]: hashed lattice values, smooth trilinear blend."""
    q = np.floor(p).astype(np.int64)
    f = p - q
    f = f * f * (3 - 2 * f)

    def h(x, y, z):
        v = (x * 73856093) ^ (y * 19349663) ^ (z * 83492791) ^ (seed * 2654435761)
        v = (v ^ (v >> 13)) * 1274126177
        v = v ^ (v >> 16)
        return (v & 0xFFFF) / 32767.5 - 1.0

    x, y, z = q[:, 0], q[:, 1], q[:, 2]
    c = [[[h(x + i, y + j, z + k) for k in (0, 1)] for j in (0, 1)] for i in (0, 1)]
    fx, fy, fz = f[:, 0], f[:, 1], f[:, 2]
    lerp = lambda a, b, t: a + (b - a) * t
    return lerp(lerp(lerp(c[0][0][0], c[0][0][1], fz), lerp(c[0][1][0], c[0][1][1], fz), fy),
                lerp(lerp(c[1][0][0], c[1][0][1], fz), lerp(c[1][1][0], c[1][1][1], fz), fy), fx)


def displaced_sphere(level: int, seed: int, amplitude: float = 0.05, freq: float = 4.0):
    """Icosphere of 20 * 4^level triangles with value-noise displacement of
    the radius; PxyzNxyzTuv attributes (normals from the displaced faces)."""
    pos, faces = grid_sphere(level)
    pos = pos * (1.0 + amplitude * value_noise(pos * freq, seed))[:, None]
    e1 = pos[faces[:, 1]] - pos[faces[:, 0]]
    e2 = pos[faces[:, 2]] - pos[faces[:, 0]]
    fn = np.cross(e1, e2)
    nrm = np.zeros_like(pos)
    for k in range(3):
        np.add.at(nrm, faces[:, k], fn)
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-20)
    uv = np.stack([0.5 + np.arctan2(pos[:, 2], pos[:, 0]) / (2 * np.pi), 0.5 - np.arcsin(np.clip(pos[:, 1], -1, 1)) / np.pi], 1)
    return np.concatenate([pos, nrm, uv], 1).astype(np.float32), faces.reshape(-1)


def _trs(rng, scale_range=(0.5, 2.0), spread=6.0):
    s = rng.uniform(*scale_range)
    a = rng.uniform(0, 2 * np.pi)
    c, si = np.cos(a), np.sin(a)
    m = np.eye(4, dtype=np.float32)
    m[0, 0], m[0, 2], m[2, 0], m[2, 2] = c * s, -si * s, si * s, c * s
    m[1, 1] = s
    m[3, 0:3] = (rng.uniform(-spread, spread), s, rng.uniform(-spread, spread))
    return m.reshape(-1)


def batch_scene(seed: int, max_bounces: int = 6) -> dict:
    """One scene of the batched configuration: a ground plane and displaced
    icospheres (instanced, random TRS with scale U[0.5, 2]) with a total
    triangle count log-uniform in [1,000, 500,000], a resolution drawn from
    {64, 128, 256, 512, 1024} squared, Ref materials (Oren-Nayar diffuse and
    glossy), a sun (directional light) and a sky colour."""
    rng = np.random.default_rng(1000 + seed)
    target = float(np.exp(rng.uniform(np.log(1e3), np.log(5e5))))
    res = int(rng.choice([64, 128, 256, 512, 1024]))
    level = int(np.clip(np.floor(np.log(target / 20.0) / np.log(4.0)), 1, 6))
    per = 20 * 4 ** level
    count = int(np.clip(round(target / per), 1, 24))
    white = np.full((1, 1, 4), 255, np.uint8)
    spec = {"textures": [(white, False, False)], "materials": [], "meshes": [], "instances": [], "size": (res, res),
            "env": {"env_col": (0.35, 0.45, 0.6)}}
    mats = spec["materials"]
    mats.append({"type": 0, "main_color": (0.5, 0.5, 0.45), "main_texture": 2, "roughness": 0.5})  # ground
    for _ in range(4):
        if rng.uniform() < 0.3:
            mats.append({"type": 1, "main_color": tuple(float(x) for x in rng.uniform(0.5, 0.95, 3)), "main_texture": 2,
                         "roughness": float(rng.uniform(0.05, 0.6))})
        else:
            mats.append({"type": 0, "main_color": tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)), "main_texture": 2,
                         "roughness": float(rng.uniform(0.0, 1.0))})
    g, gi = _quad((-40, 0, -40), (-40, 0, 40), (40, 0, 40), (40, 0, -40), (0, 1, 0))
    spec["meshes"].append((g, gi, [(0, 0, 0, 6)], 0))
    spec["instances"].append((0, np.eye(4, dtype=np.float32).reshape(-1)))
    n_meshes = min(count, 3)
    for m in range(n_meshes):
        a, i = displaced_sphere(level, seed * 7 + m)
        mat = 1 + m % 4
        spec["meshes"].append((a, i, [(mat, mat, 0, len(i))], 0))
    for k in range(count):
        spec["instances"].append((1 + k % n_meshes, _trs(rng)))
    sun = rng.normal(size=3)
    sun[1] = -abs(sun[1]) - 1.0
    spec["lights"] = [{"type": 2, "position": (0.0, 0.0, 0.0), "radius": 0.0, "color": (2.5, 2.4, 2.2),
                       "direction": tuple(float(x) for x in sun / np.linalg.norm(sun)), "angle": 1.0}]
    spec["camera"] = {"type": 0, "filter": 1, "dtype": 0, "origin": (0.0, 9.0, -16.0), "fwd": (0.0, -0.45, 0.9), "up": (0.0, 1.0, 0.0),
                      "fov": 55.0, "gamma": 1.0, "max_total_depth": max_bounces, "max_diff_depth": max_bounces,
                      "max_glossy_depth": max_bounces, "termination_start_depth": 3}
    spec["tris"] = 2 + count * per
    return spec


# ------------------------------------------------ metallic-roughness atrium

def _wall(corners, n, uv_scale):
    """A quad with normal n (winding fixed to agree with it) and UVs tiled uv_scale times."""
    p = [np.asarray(c, np.float64) for c in corners]
    if np.dot(np.cross(p[1] - p[0], p[2] - p[0]), n) < 0:
        p = p[::-1]
    a, i = _quad(*p, n)
    a[:, 6:8] *= np.asarray(uv_scale, np.float32)
    return a, i


def noise_texture(res: int, seed: int) -> np.ndarray:
    """res x res RGBA8 albedo from two octaves of value noise (tileable only
    in the sense that sampling wraps)."""
    y, x = np.meshgrid(np.arange(res), np.arange(res), indexing="ij")
    p = np.stack([x.reshape(-1) / res, y.reshape(-1) / res, np.zeros(res * res)], 1)
    n = 0.65 * value_noise(p * 12.0, seed) + 0.35 * value_noise(p * 48.0 + 7.0, seed + 1)
    rgb = np.stack([0.55 + 0.30 * n, 0.50 + 0.25 * n, 0.42 + 0.20 * n], 1)
    img = np.empty((res * res, 4), np.uint8)
    img[:, :3] = np.clip(np.round(rgb * 255.0), 0, 255).astype(np.uint8)
    img[:, 3] = 255
    return img.reshape(res, res, 4)


def atrium(seed: int = 0, w: int = 1280, h: int = 720, max_bounces: int = 8, level: int = 5, n_spheres: int = 16,
           tex_res: int = 1024, room=(20.0, 4.0, 60.0), n_materials: int | None = None) -> dict:
    """The metallic-roughness render configuration: a closed box room of
    room[0] x room[1] x room[2] (12 triangles, seen from inside) and
    n_spheres displaced icospheres of 20 * 4^level triangles each (value-noise
    displacement of amplitude 0.05), each its own mesh placed by one instance
    with a random TRS (scale U[0.5, 2], rotation about y). Every material is
    RAY_MAT_PRINCIPLED with roughness U[0.05, 1], metallic Bernoulli(0.3) and
    its albedo from one tex_res^2 RGBA8 value-noise texture (tinted per
    material). Lights: a sun of irradiance 5 (outside the closed room, so its
    shadow rays are all blocked) and 4 quad lights under the ceiling. All
    surfaces are two-sided. n_materials (optional): that many materials in
    all, the room taking the first and the spheres the others in turn."""
    rng = np.random.default_rng(2000 + seed)
    X, Y, Z = (float(v) for v in room)
    spec = {"textures": [(noise_texture(tex_res, seed), True, False)], "materials": [], "meshes": [], "instances": [], "lights": [],
            "env": {"env_col": (0.0, 0.0, 0.0)}}
    mats = spec["materials"]

    def material(tint):
        mats.append({"type": 6, "main_color": tuple(float(c) for c in tint), "main_texture": 2, "roughness": float(rng.uniform(0.05, 1.0)),
                     "metallic": float(rng.uniform() < 0.3)})
        return len(mats) - 1

    # the room: floor, ceiling and four walls, normals pointing inwards
    m_room = material((1.0, 1.0, 1.0))
    hx, hz = X / 2.0, Z / 2.0
    walls = [
        ([(-hx, 0, -hz), (hx, 0, -hz), (hx, 0, hz), (-hx, 0, hz)], (0, 1, 0), (X / 4, Z / 4)),
        ([(-hx, Y, -hz), (-hx, Y, hz), (hx, Y, hz), (hx, Y, -hz)], (0, -1, 0), (X / 4, Z / 4)),
        ([(-hx, 0, -hz), (-hx, 0, hz), (-hx, Y, hz), (-hx, Y, -hz)], (1, 0, 0), (Z / 4, Y / 4)),
        ([(hx, 0, -hz), (hx, Y, -hz), (hx, Y, hz), (hx, 0, hz)], (-1, 0, 0), (Z / 4, Y / 4)),
        ([(-hx, 0, -hz), (-hx, Y, -hz), (hx, Y, -hz), (hx, 0, -hz)], (0, 0, 1), (X / 4, Y / 4)),
        ([(-hx, 0, hz), (hx, 0, hz), (hx, Y, hz), (-hx, Y, hz)], (0, 0, -1), (X / 4, Y / 4)),
    ]
    parts = [(*_wall(c, np.asarray(n, np.float64), s), m_room) for c, n, s in walls]
    a, i, shapes = _concat(parts)
    spec["meshes"].append((a, i, shapes, 0))
    spec["instances"].append((0, np.eye(4, dtype=np.float32).reshape(-1)))
    sphere_mats = None
    if n_materials is not None:
        sphere_mats = [material(rng.uniform(0.5, 1.0, 3)) for _ in range(max(1, n_materials - 1))]
    for k in range(n_spheres):
        m = material(rng.uniform(0.5, 1.0, 3)) if sphere_mats is None else sphere_mats[k % len(sphere_mats)]
        a, i = displaced_sphere(level, seed * 101 + k, amplitude=0.05)
        spec["meshes"].append((a, i, [(m, m, 0, len(i))], 0))
        s = rng.uniform(0.5, 2.0)
        ang = rng.uniform(0, 2 * np.pi)
        c, si = np.cos(ang), np.sin(ang)
        xf = np.eye(4, dtype=np.float32)
        xf[0, 0], xf[0, 2], xf[2, 0], xf[2, 2] = c * s, -si * s, si * s, c * s
        xf[1, 1] = s
        xf[3, 0:3] = (rng.uniform(-hx + 1.5, hx - 1.5), min(s, Y / 2), rng.uniform(-hz + 3.0, hz - 3.0))
        spec["instances"].append((k + 1, xf.reshape(-1)))
    sun = np.array([0.35, -1.0, 0.25])
    spec["lights"].append({"type": 4, "color": (5.0, 5.0, 5.0), "direction": tuple(float(v) for v in sun / np.linalg.norm(sun)),
                           "angle": 0.53})
    for k in range(4):
        z = -hz + Z * (k + 0.5) / 4.0
        spec["lights"].append({"type": 3, "position": (-1.5, Y - 0.01, z - 1.5), "color": (30.0, 28.5, 26.0), "edge_u": (3.0, 0.0, 0.0),
                               "edge_v": (0.0, 0.0, 3.0)})
    spec["camera"] = {"type": 0, "filter": 1, "dtype": 0, "origin": (0.0, Y * 0.5, -hz + 1.0), "fwd": (0.0, -0.04, 1.0),
                      "up": (0.0, 1.0, 0.0), "fov": 60.0, "gamma": 1.0, "max_total_depth": max_bounces, "max_diff_depth": max_bounces,
                      "max_glossy_depth": max_bounces, "termination_start_depth": 3}
    spec["size"] = (w, h)
    spec["tris"] = 12 + n_spheres * 20 * 4 ** level
    return spec


def float_noise_texture(res: int, seed: int) -> np.ndarray:
    """res x res x 3 float32 albedo in [0.15, 0.85] from two octaves of value noise."""
    y, x = np.meshgrid(np.arange(res), np.arange(res), indexing="ij")
    p = np.stack([x.reshape(-1) / res, y.reshape(-1) / res, np.zeros(res * res)], 1)
    chans = []
    for c in range(3):
        n = 0.65 * value_noise(p * 10.0 + 3.0 * c, seed + 11 * c) + 0.35 * value_noise(p * 40.0 + 5.0 * c, seed + 11 * c + 1)
        chans.append(0.5 + 0.35 * n)
    return np.clip(np.stack(chans, 1), 0.0, 1.0).astype(np.float32).reshape(res, res, 3)


def diff_atrium(seed: int = 0, w: int = 256, h: int = 256, max_bounces: int = 4, level: int = 5, n_spheres: int = 16,
                tex_res: int = 512, n_materials: int = 8) -> dict:
    """The differentiable configuration: the atrium with n_materials materials
    (every one differentiable, material k in roughness slot k) seen at w x h,
    max_bounces bounces and no Russian roulette (termination starts at the
    last bounce). Hidden parameters: a tex_res^2 RGB value-noise albedo and
    roughness U[0.1, 0.9] per material. Returns the scene spec with the keys
    'albedo_target' (tex_res, tex_res, 3), 'rough_target' (n_materials,) and
    'material_slot'."""
    spec = atrium(seed, w, h, max_bounces, level=level, n_spheres=n_spheres, tex_res=64, n_materials=n_materials)
    rng = np.random.default_rng(3000 + seed)
    spec["camera"] = dict(spec["camera"], termination_start_depth=max_bounces)
    spec["albedo_target"] = float_noise_texture(tex_res, seed + 17)
    spec["rough_target"] = rng.uniform(0.1, 0.9, len(spec["materials"])).astype(np.float32)
    spec["material_slot"] = list(range(len(spec["materials"])))
    return spec
