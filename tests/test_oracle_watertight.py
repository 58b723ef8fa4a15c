"""The oracle's watertight ray/triangle test (a restatement of Woop, Benthin and Wald,
"Watertight Ray/Triangle Intersection", JCGT 2013; the reference has no such mode: its
rayTriangle, src/bvh/bvh_traverse.cpp:47-87, culls back faces) checked by the properties the
paper proves, so that the GPU's RT_TRACE_WATERTIGHT mode, tested against it bit for bit in
test_gpu_trace.py, rests on an independent check:

* no ray through a closed mesh leaks: rays aimed exactly at every vertex and every edge
  midpoint of a closed icosphere, from outside and from inside, all hit it;
* both faces count: from inside a closed mesh the watertight test hits where the reference's
  culling test sees only back faces;
* where the reference's test hits a front face, the watertight test finds the same nearest
  distance to float rounding."""
import numpy as np

from oracle import Baked, VARIANTS, make_cfg
from rtb200 import scenes

WATERTIGHT, ANY_HIT = 2, 1


def closed_sphere(level=3):
    v, t = scenes.icosphere(level, radius=1.0, disp=0.0)
    return v, t


def targets(v, t):
    """Every vertex and every edge midpoint of the mesh (float32 positions)."""
    p = v[:, :3].astype(np.float64)
    edges = np.unique(np.sort(np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]]), axis=1), axis=0)
    return np.concatenate([p, 0.5 * (p[edges[:, 0]] + p[edges[:, 1]])])


def rays_at(points, origin_fn):
    o = origin_fn(points)
    d = points - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((points.shape[0], 8), np.float32)
    r[:, 0:3] = o; r[:, 3] = 0.0; r[:, 4:7] = d; r[:, 7] = np.inf
    return r


def test_no_leaks_through_vertices_and_edges(orc):
    """The triangle test alone (every ray against every triangle): a leak here would be the
    test's own. Through a BVH a ray aimed exactly at a vertex on a node's box face can still
    miss the box (the reference's slab test is not conservative), which the paper leaves to
    the traversal."""
    v, t = closed_sphere()
    pts = targets(v, t)
    for name, origin in (("outside", lambda p: 3.0 * p), ("inside", lambda p: np.zeros_like(p)),
                         ("off-centre inside", lambda p: np.tile([0.11, -0.07, 0.05], (p.shape[0], 1)))):
        rays = rays_at(pts, origin)
        for flags in (WATERTIGHT, WATERTIGHT | ANY_HIT):
            h, _, _ = orc.trace_brute(v, t, rays, flags=flags)
            assert h.all(), f"{name}: {int((h == 0).sum())} of {h.size} rays leaked (flags {flags})"
        if name == "outside":
            # the reference's Moller-Trumbore test does leak through some of these edges and
            # vertices (about one ray in nine on this mesh): the contrast the mode exists for
            h_mt, _, _ = orc.trace_brute(v, t, rays, flags=0)
            assert 0.5 < h_mt.mean() < 1.0


def test_both_faces_from_inside(orc):
    v, t = closed_sphere(2)
    baked = orc.build(v, t, make_cfg(**VARIANTS["lbvh63"]))
    rays = scenes.incoherent_rays(5000, [-0.2] * 3, [0.2] * 3, seed=3)
    h_cull, _, _, _, _ = orc.trace(baked, rays, flags=0, threads=4)
    h_wt, out, _, _, _ = orc.trace(baked, rays, flags=WATERTIGHT, threads=4)
    assert h_cull.sum() == 0 and h_wt.all()
    # the hit lies on the sphere of radius 1 (to its tessellation)
    p = rays[:, 0:3] + rays[:, 4:7] * out[:, 0:1]
    r = np.linalg.norm(p, axis=1)
    assert np.all((r > 0.9) & (r < 1.0 + 1e-5))


def test_front_faces_agree_with_the_reference_test(orc):
    v, t = scenes.soup(3000, seed=31)
    baked = orc.build(v, t, make_cfg(**VARIANTS["sah4"]))
    rays = scenes.incoherent_rays(20000, [0.0] * 3, [1.0] * 3, seed=32)
    h0, o0, t0, _, _ = orc.trace(baked, rays, flags=0, threads=4)
    h1, o1, t1, _, _ = orc.trace(baked, rays, flags=WATERTIGHT, threads=4)
    assert np.all(h1[h0 == 1] == 1)  # the culling test's hits are a subset
    both = (h0 == 1) & (t0 == t1)
    assert both.sum() >= 0.99 * (h0 == 1).sum()
    assert np.allclose(o1[both, 0], o0[both, 0], rtol=2e-6, atol=0)
    assert np.allclose(o1[both, 1:3], o0[both, 1:3], atol=2e-4)  # barycentrics by another formula
