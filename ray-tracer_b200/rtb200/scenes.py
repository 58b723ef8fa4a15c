"""Seeded synthetic scenes for the benchmark workloads and the parity tests.

All geometry is float32 in the reference's vertex layout (x, y, z, nx, ny, nz) with
uint32 triangle index triples. The generators are pinned here in code so that the GPU
build, the oracle and the CPU baseline all see identical inputs.

* ``soup``       -- the BVH microbenchmark soup: N triangles, centroid uniform in [0,1]^3,
                    each vertex at centroid + L * u with L log-uniform in [1e-4, 1e-2] and u
                    uniform on the unit sphere (one independent draw per vertex).
* ``icosphere``  -- icosahedron subdivided ``level`` times (20 * 4**level triangles, shared
                    vertices), each vertex pushed radially by uniform[-disp, disp] * radius.
* ``cornell``    -- a Cornell box of 5 axis-aligned quads (2 triangles each) facing inward
                    plus one quad area light under the ceiling, facing down.
* ``incoherent_rays`` / ``pinhole_rays`` -- the microbenchmark ray sets.
"""
from __future__ import annotations

import numpy as np

BASE_SEED = 20261203


def _face_normals(v, t):
    p0, p1, p2 = v[t[:, 0], :3], v[t[:, 1], :3], v[t[:, 2], :3]
    n = np.cross(p1 - p0, p2 - p0)
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    return n / np.maximum(ln, 1e-30)


def soup(n: int, seed: int = BASE_SEED + 1, lo: float = 1e-4, hi: float = 1e-2):
    """Random triangle soup; returns (verts (3n, 6) f32, tris (n, 3) u32)."""
    rng = np.random.default_rng(seed)
    c = rng.random((n, 1, 3), dtype=np.float64)
    L = np.exp(rng.uniform(np.log(lo), np.log(hi), size=(n, 3, 1)))
    u = rng.normal(size=(n, 3, 3))
    u /= np.linalg.norm(u, axis=2, keepdims=True)
    p = (c + L * u).reshape(-1, 3).astype(np.float32)
    tris = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    verts = np.zeros((3 * n, 6), np.float32)
    verts[:, :3] = p
    fn = _face_normals(verts, tris).astype(np.float32)
    verts[:, 3:] = np.repeat(fn, 3, axis=0)
    return verts, tris


def _icosahedron():
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    return v, f


_SUBDIV = {}


def _subdivided(level: int):
    """Unit icosphere after ``level`` midpoint subdivisions (cached)."""
    if level in _SUBDIV:
        return _SUBDIV[level]
    v, f = _icosahedron()
    for _ in range(level):
        cache = {}
        verts = list(v)

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                m = m / np.linalg.norm(m)
                cache[key] = len(verts)
                verts.append(m)
            return cache[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        v = np.array(verts)
        f = np.array(nf, np.int64)
    _SUBDIV[level] = (v, f)
    return v, f


def icosphere(level: int, center=(0.0, 0.0, 0.0), radius: float = 1.0, disp: float = 0.05,
              seed: int = BASE_SEED, max_tris: int | None = None):
    """Displaced icosphere; outward-facing under the reference's winding convention.

    ``max_tris`` keeps the first faces of the subdivided mesh (the truncation rule of the
    50,000- and 12,500-triangle variants); unreferenced vertices are kept."""
    v, f = _subdivided(level)
    rng = np.random.default_rng(seed)
    scale = 1.0 + rng.uniform(-disp, disp, size=(v.shape[0], 1))
    p = v * scale * radius + np.asarray(center, np.float64)
    if max_tris is not None:
        f = f[:max_tris]
    # The reference culls triangles whose geometric normal faces along the ray
    # (src/bvh/bvh_traverse.cpp:57 rejects dot(e1, cross(d, e2)) >= 0), so a surface seen
    # from outside must be wound clockwise as seen from outside: flip the icosahedron's
    # counter-clockwise faces.
    f = f[:, [0, 2, 1]]
    verts = np.zeros((v.shape[0], 6), np.float32)
    verts[:, :3] = p.astype(np.float32)
    # smooth normals: area-weighted face normals accumulated per vertex (outward)
    fp = p[f]
    fn = np.cross(fp[:, 2] - fp[:, 0], fp[:, 1] - fp[:, 0])
    acc = np.zeros_like(p)
    for k in range(3):
        np.add.at(acc, f[:, k], fn)
    ln = np.linalg.norm(acc, axis=1, keepdims=True)
    acc = np.where(ln > 0, acc / np.maximum(ln, 1e-30), v)
    verts[:, 3:] = acc.astype(np.float32)
    return verts, np.ascontiguousarray(f, dtype=np.uint32)


def quad(p0, p1, p2, p3, normal):
    """Two triangles (p0, p1, p2) and (p0, p2, p3); wound so that rays travelling against
    ``normal`` hit them under the reference's culling rule."""
    P = np.array([p0, p1, p2, p3], np.float64)
    n = np.asarray(normal, np.float64)
    e1, e2 = P[1] - P[0], P[2] - P[0]
    # accepted iff dot(e1, cross(d, e2)) < 0 for d = -n  <=>  dot(cross(e1, e2), n) < 0
    if np.dot(np.cross(e1, e2), n) > 0:
        P = P[[0, 3, 2, 1]]
    verts = np.zeros((4, 6), np.float32)
    verts[:, :3] = P.astype(np.float32)
    verts[:, 3:] = (n / np.linalg.norm(n)).astype(np.float32)
    tris = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    return verts, tris


def cornell(size: float = 2.0, light_size: float = 0.5):
    """Cornell box spanning [-size/2, size/2]^3 with an open front (z = -size/2); returns
    (verts, tris, object id per triangle) with object ids 0 floor, 1 ceiling, 2 back,
    3 left, 4 right, 5 light."""
    h = size / 2.0
    walls = [
        ([-h, -h, -h], [h, -h, -h], [h, -h, h], [-h, -h, h], [0, 1, 0]),     # floor
        ([-h, h, -h], [h, h, -h], [h, h, h], [-h, h, h], [0, -1, 0]),       # ceiling
        ([-h, -h, h], [h, -h, h], [h, h, h], [-h, h, h], [0, 0, -1]),       # back
        ([-h, -h, -h], [-h, -h, h], [-h, h, h], [-h, h, -h], [1, 0, 0]),    # left
        ([h, -h, -h], [h, -h, h], [h, h, h], [h, h, -h], [-1, 0, 0]),       # right
    ]
    l = light_size / 2.0
    y = h - 1e-3 * size
    walls.append(([-l, y, -l], [l, y, -l], [l, y, l], [-l, y, l], [0, -1, 0]))
    return concat([quad(*w) for w in walls])


def concat(parts):
    """Concatenate (verts, tris) parts; returns (verts, tris, part id per triangle)."""
    vs, ts, ids = [], [], []
    off = 0
    for i, (v, t) in enumerate(parts):
        vs.append(v)
        ts.append(t.astype(np.uint64) + off)
        ids.append(np.full(t.shape[0], i, np.uint32))
        off += v.shape[0]
    return (np.concatenate(vs).astype(np.float32), np.concatenate(ts).astype(np.uint32),
            np.concatenate(ids))


def incoherent_rays(n: int, lo, hi, seed: int = BASE_SEED + 7, tmin: float = 0.0, tmax: float = np.inf):
    """Origins uniform in the box [lo, hi], directions uniform on S^2; (n, 8) f32."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(np.asarray(lo, np.float64), np.asarray(hi, np.float64), size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.empty((n, 8), np.float32)
    r[:, 0:3] = o; r[:, 3] = tmin; r[:, 4:7] = d; r[:, 7] = tmax
    return r


def pinhole_rays(width: int, height: int, pos, target, fov_deg: float = 60.0):
    """One primary ray per pixel centre of a look-at pinhole camera; (W*H, 8) f32."""
    pos = np.asarray(pos, np.float64); target = np.asarray(target, np.float64)
    fwd = target - pos; fwd /= np.linalg.norm(fwd)
    up0 = np.array([0.0, 1.0, 0.0]) if abs(fwd[1]) < 0.99 else np.array([1.0, 0.0, 0.0])
    right = np.cross(fwd, up0); right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    th = np.tan(np.radians(fov_deg) * 0.5)
    aspect = width / height
    xs = ((np.arange(width) + 0.5) / width * 2 - 1) * aspect * th
    ys = ((np.arange(height) + 0.5) / height * 2 - 1) * th
    X, Y = np.meshgrid(xs, ys)
    d = fwd[None, None, :] + X[..., None] * right + Y[..., None] * up
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    r = np.empty((width * height, 8), np.float32)
    r[:, 0:3] = pos; r[:, 3] = 1e-3; r[:, 4:7] = d.reshape(-1, 3); r[:, 7] = np.inf
    return r


# ---- benchmark scenes ---------------------------------------------------------------------

class Scene:
    """Geometry plus shading: obj = object id per input triangle, mats = material dicts,
    mat_of_obj = material per object, lookat = (pos, target, fov_deg)."""

    def __init__(self, verts, tris, obj, mats, mat_of_obj, lookat, env_kind=1, env_color=(0.0, 0.0, 0.0)):
        self.verts, self.tris, self.obj = verts, tris, np.asarray(obj, np.uint32)
        self.mats, self.mat_of_obj = mats, np.asarray(mat_of_obj, np.uint32)
        self.lookat, self.env_kind, self.env_color = lookat, env_kind, env_color

    @property
    def mat_of_tri(self):
        """material per input triangle"""
        return self.mat_of_obj[self.obj]

    def baked_materials(self, prim_ids):
        """material per baked triangle, from the build's original-triangle ids"""
        return self.mat_of_tri[np.asarray(prim_ids, np.int64)]


CORNELL_LOOKAT = ((0.0, 0.0, -3.4), (0.0, 0.0, 0.0), 40.0)


def _cornell_parts(light_radiance=15.0):
    """(verts, tris, obj) of the box and the light (objects 0-5) and its 6 materials."""
    cv, ct, cid = cornell()
    mats = [dict(albedo=(0.75, 0.75, 0.75)), dict(albedo=(0.75, 0.75, 0.75)), dict(albedo=(0.75, 0.75, 0.75)),
            dict(albedo=(0.65, 0.1, 0.1)), dict(albedo=(0.1, 0.6, 0.15)),
            dict(albedo=(0.0, 0.0, 0.0), emission=(light_radiance,) * 3)]
    return cv, ct, cid, mats


def plain_scene(seed: int = BASE_SEED, sphere_tris=None):
    """The plain path-tracing workload: the Cornell box (5 quads and a quad light of radiance
    15), an icosphere subdivided 5 times (20,480 triangles, vertices displaced radially by
    uniform[-0.05, 0.05]) and two spheres of radius 0.3 from the reference's addSphere
    (16 rings x 32 sectors), all Lambertian with albedo uniform[0.2, 0.8] per object.
    sphere_tris: (verts, tris) of one reference sphere at the origin (rtb200.Mesh), passed in
    so this module needs no library."""
    cv, ct, cid, mats = _cornell_parts()
    iv, it = icosphere(5, center=(0.15, -0.45, 0.25), radius=0.5, seed=seed)
    parts = [(cv, ct), (iv, it)]
    if sphere_tris is not None:
        for c in ((-0.55, -0.7, -0.35), (0.6, -0.7, -0.5)):
            v = sphere_tris[0].copy()
            v[:, :3] += np.asarray(c, np.float32)
            parts.append((v, sphere_tris[1]))
    v, t, part = concat(parts)
    obj = np.where(part == 0, cid[np.minimum(np.arange(t.shape[0]), ct.shape[0] - 1)], 5 + part).astype(np.uint32)
    rng = np.random.default_rng(seed + 1)
    n_obj = 6 + len(parts) - 1
    for _ in range(6, n_obj):
        a = rng.uniform(0.2, 0.8)
        mats.append(dict(albedo=(a, a, a)))
    # one albedo per object: the box's own walls keep their Cornell colours
    return Scene(v, t, obj, mats, np.arange(n_obj), CORNELL_LOOKAT)


def diff_scene(n_ico_tris: int = 50000, seed: int = BASE_SEED + 3):
    """The differentiable-rendering workload: the Cornell box and a displaced icosphere
    subdivided as few times as give n_ico_tris faces (6 times for 50,000) truncated to its first
    n_ico_tris faces. Returns (Scene, init albedo, ground-truth albedo) with RGB albedos per
    input triangle, uniform[0.2, 0.8]."""
    cv, ct, cid, mats = _cornell_parts()
    level = 0
    while 20 * 4 ** level < n_ico_tris:
        level += 1
    iv, it = icosphere(level, center=(0.0, -0.35, 0.2), radius=0.55, seed=seed, max_tris=n_ico_tris)
    v, t, part = concat([(cv, ct), (iv, it)])
    obj = np.concatenate([cid, np.full(it.shape[0], 6, np.uint32)])
    mats = mats + [dict(albedo=(0.5, 0.5, 0.5))]
    rng = np.random.default_rng(seed + 1)
    init = rng.uniform(0.2, 0.8, size=(t.shape[0], 3)).astype(np.float32)
    gt = rng.uniform(0.2, 0.8, size=(t.shape[0], 3)).astype(np.float32)
    for alb in (init, gt):      # the box keeps its colours; the light is black
        alb[:ct.shape[0]] = np.array([mats[o]["albedo"] for o in cid], np.float32)
    return Scene(v, t, obj, mats, np.arange(7), CORNELL_LOOKAT), init, gt


def large_scene(n_spheres: int = 400, tris_per_sphere: int = 12500, seed: int = BASE_SEED + 4):
    """The large-render workload: n_spheres displaced icospheres (subdivided 6 times, first
    tris_per_sphere faces) placed uniformly in the unit box with scale log-uniform in
    [0.01, 0.2], 80 % Lambertian (albedo uniform[0.2, 0.8]) / 20 % mirror, a floor and 4 quad
    area lights above. Camera outside the box."""
    rng = np.random.default_rng(seed)
    level = 5 if tris_per_sphere <= 20480 else 6
    parts, objs, mats = [], [], []
    for i in range(n_spheres):
        c = rng.uniform(0.0, 1.0, size=3)
        r = float(np.exp(rng.uniform(np.log(0.01), np.log(0.2))))
        v, t = icosphere(level, center=c, radius=r, seed=seed + 100 + i, max_tris=tris_per_sphere)
        parts.append((v, t))
        if rng.uniform() < 0.2:
            mats.append(dict(albedo=(0.9, 0.9, 0.9), kind=1))
        else:
            a = rng.uniform(0.2, 0.8, size=3)
            mats.append(dict(albedo=tuple(float(x) for x in a)))
    fv, ft = quad((-1.0, -0.05, -1.0), (2.0, -0.05, -1.0), (2.0, -0.05, 2.0), (-1.0, -0.05, 2.0), (0, 1, 0))
    parts.append((fv, ft)); mats.append(dict(albedo=(0.6, 0.6, 0.6)))
    for k, (lx, lz) in enumerate(((0.15, 0.15), (0.85, 0.15), (0.15, 0.85), (0.85, 0.85))):
        lv, lt = quad((lx - 0.1, 1.6, lz - 0.1), (lx + 0.1, 1.6, lz - 0.1), (lx + 0.1, 1.6, lz + 0.1),
                      (lx - 0.1, 1.6, lz + 0.1), (0, -1, 0))
        parts.append((lv, lt))
        mats.append(dict(albedo=(0.0, 0.0, 0.0), emission=(20.0, 18.0 + 2 * k, 16.0)))
    v, t, part = concat(parts)
    return Scene(v, t, part, mats, np.arange(len(parts)), ((0.5, 0.9, -1.6), (0.5, 0.35, 0.5), 45.0),
                 env_kind=1, env_color=(0.02, 0.02, 0.03))


def batch_scene(n_tris: int, seed: int):
    """One scene of the batched workload: a displaced icosphere (the smallest subdivision with
    n_tris faces, truncated to them) or a triangle soup of n_tris triangles in the unit box
    (even / odd seed), a floor and one quad area light above, all Lambertian, object albedo
    uniform[0.2, 0.8]."""
    rng = np.random.default_rng(seed)
    if seed % 2 == 0:
        level = 0
        while 20 * 4 ** level < n_tris:
            level += 1
        ov, ot = icosphere(level, center=(0.5, 0.45, 0.5), radius=0.4, seed=seed, max_tris=n_tris)
    else:
        ov, ot = soup(n_tris, seed=seed)
    fv, ft = quad((-1.0, -0.05, -1.0), (2.0, -0.05, -1.0), (2.0, -0.05, 2.0), (-1.0, -0.05, 2.0), (0, 1, 0))
    lv, lt = quad((0.3, 1.5, 0.3), (0.7, 1.5, 0.3), (0.7, 1.5, 0.7), (0.3, 1.5, 0.7), (0, -1, 0))
    v, t, part = concat([(ov, ot), (fv, ft), (lv, lt)])
    a = rng.uniform(0.2, 0.8, size=3)
    mats = [dict(albedo=tuple(float(x) for x in a)), dict(albedo=(0.5, 0.5, 0.5)),
            dict(albedo=(0.0, 0.0, 0.0), emission=(12.0, 12.0, 12.0))]
    return Scene(v, t, part, mats, np.arange(3), ((0.5, 0.9, -1.4), (0.5, 0.4, 0.5), 45.0))


def batch_scenes(n_scenes: int = 64, lo: int = 1000, hi: int = 500000, seed: int = BASE_SEED + 2):
    """The batched workload: n_scenes scenes with triangle counts log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), size=n_scenes)).astype(np.int64)
    return [batch_scene(int(c), seed + 1 + i) for i, c in enumerate(counts)]


def batch_shading(scs):
    """Materials of a list of scenes concatenated, and the material of every input triangle
    of the concatenated batch."""
    mats, mot, off = [], [], 0
    for sc in scs:
        mats += sc.mats
        mot.append(sc.mat_of_tri + off)
        off += len(sc.mats)
    return mats, np.concatenate(mot).astype(np.uint32)
