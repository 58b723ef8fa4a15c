"""Pins the oracle (the C restatement in oracle/rt_oracle.c) before anything is checked against it:

* against the golden fixtures in tests/golden/ (made by running the reference itself,
  tests/golden/make_golden.py) -- runs anywhere;
* against the reference compiled from its own sources (oracle/_ref, oracle/build_ref.sh),
  bit for bit, on seeded scenes for every build variant, on traces, on Morton codes, on the
  normal renormalisation and on triangle clipping -- where oracle/_ref was built;
* against the known answers of the reference's tests/test_traverse.cpp (12 rays) and
  tests/test_aabb.cpp (clipping cases).
Runs on the CPU (no GPU needed).
"""
import glob
import os
import tempfile

import numpy as np
import pytest

import oracle
from oracle import VARIANTS, Baked, Reference, make_cfg
from rtb200 import scenes
from scenes_for_tests import TEST_TRAVERSE_SCN, big_and_small, identical, planar

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def same_tree(a: Baked, b: Baked):
    assert a.nodes.shape == b.nodes.shape
    for f in ("is_leaf", "a", "b"):
        assert np.array_equal(a.nodes[f], b.nodes[f]), f
    for f in ("bmin", "bmax"):
        assert np.array_equal(a.nodes[f].view(np.uint32), b.nodes[f].view(np.uint32)), f
    assert np.array_equal(a.tris, b.tris)
    assert np.array_equal(a.verts.view(np.uint32), b.verts.view(np.uint32))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_restatement_matches_golden(orc, path):
    g = np.load(path)
    variant = os.path.basename(path)[:-4].split("_")[-1]
    b = orc.build(g["verts"], g["tris"], make_cfg(**VARIANTS[variant]))
    same_tree(b, Baked(g["nodes"].view(oracle.NODE_DTYPE), g["btris"], g["bverts"]))
    hit, out, tri, _, of = orc.trace(b, g["rays"])
    assert of == 0
    assert np.array_equal(hit, g["hit"])
    m = hit == 1
    assert np.array_equal(tri[m], g["tri"][m])
    assert np.array_equal(out[m].view(np.uint32), g["out"][m].view(np.uint32))
    codes, perm, sbox = orc.morton(g["verts"], g["tris"], make_cfg(**VARIANTS[variant]))
    assert np.array_equal(codes, g["codes"]) and np.array_equal(perm, g["perm"])
    assert np.array_equal(sbox, g["scene_box"])


needs_ref = pytest.mark.skipif(not Reference.available("hybrid"), reason="oracle/_ref not built")


def _scenes():
    return {
        "soup3k": scenes.soup(3000, seed=41),
        "ico3": scenes.icosphere(3, seed=42),
        "identical64": identical(64, seed=43),
        "planar300": planar(300, seed=44),
        "big_small": big_and_small(1500, seed=45),
        "one": scenes.soup(1, seed=46),
    }


@needs_ref
@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_restatement_matches_reference_bake(orc, variant):
    ref = Reference(variant)
    consts = ref.constants()
    kw = VARIANTS[variant]
    assert consts[0] == min(kw["lbvh_threshold"], 2147483647) and consts[1] == kw["max_leaf"]
    assert consts[2] == kw["morton_bits"] and consts[5] == 48
    for name, (v, t) in _scenes().items():
        same_tree(orc.build(v, t, make_cfg(**kw)), ref.bake(v, t))


@needs_ref
def test_restatement_matches_reference_trace(orc):
    ref = Reference("hybrid")
    v, t = big_and_small(2000, seed=47)
    b = ref.bake(v, t)
    lo, hi = v[:, :3].min(0), v[:, :3].max(0)
    rays = scenes.incoherent_rays(20000, lo - 0.1, hi + 0.1, seed=48)
    rays[:2000, 4:7] = 0.0  # axis-parallel rays: NaN slabs
    rays[np.arange(2000), 4 + np.arange(2000) % 3] = 1.0
    h1, o1, t1 = ref.trace(b, rays, threads=4)
    h2, o2, t2, _, _ = orc.trace(b, rays, threads=4)
    assert np.array_equal(h1, h2)
    m = h1 == 1
    assert np.array_equal(t1[m], t2[m]) and np.array_equal(o1[m].view(np.uint32), o2[m].view(np.uint32))


@needs_ref
def test_restatement_matches_reference_morton_and_normals(orc):
    ref = Reference("lbvh30")
    v, t = scenes.soup(5000, seed=49)
    c1, p1, s1 = ref.morton(v, t)
    c2, p2, s2 = orc.morton(v, t, make_cfg(**VARIANTS["lbvh30"]))
    assert np.array_equal(c1, c2) and np.array_equal(p1, p2) and np.array_equal(s1, s2)
    # normal renormalisation incl. tiny and zero normals (bvh_IO.cpp:102-118)
    rng = np.random.default_rng(50)
    w = v.copy()
    w[:, 3:] = rng.normal(size=(w.shape[0], 3)).astype(np.float32) * np.float32(10.0) ** rng.integers(-8, 8, (w.shape[0], 1))
    w[:10, 3:] = 0.0
    a = ref.init_geos(w, t)
    b = orc.normalize_normals(w)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@needs_ref
def test_clip_triangle_matches_reference(orc):
    ref = Reference("hybrid")
    rng = np.random.default_rng(51)
    for _ in range(3000):
        v9 = rng.uniform(-2, 2, 9).astype(np.float32)
        lo = rng.uniform(-1.5, 0.5, 3)
        box6 = np.concatenate([lo, lo + rng.uniform(0.01, 2.0, 3)]).astype(np.float32)
        a, b = ref.clip_triangle(v9, box6), orc.clip_triangle(v9, box6)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_clip_triangle_known_answers(orc):
    """Cases of the reference's tests/test_aabb.cpp (clipTriangleToAABB suite)."""
    box = np.array([0, 0, 0, 4, 4, 4], np.float32)
    inside = orc.clip_triangle(np.array([1, 1, 1, 3, 1, 1, 1, 3, 1], np.float32), box)
    assert np.allclose(inside, [1, 1, 1, 3, 3, 1])
    outside = orc.clip_triangle(np.array([5, 5, 5, 6, 5, 5, 5, 6, 5], np.float32), box)
    assert outside[0] > outside[3]  # empty box
    straddle = orc.clip_triangle(np.array([-2, 1, 1, 2, 1, 1, 0, 3, 1], np.float32), box)
    assert np.allclose(straddle[[0, 3]], [0, 2]) and straddle[1] == 1 and straddle[4] <= 3


TRAVERSE_RAYS = [  # tests/test_traverse.cpp:117-236: origin, direction, hit?, t range, normal axis, sign
    ((0, 0, 0), (0, 0, 1), True, (3.9, 4.1), 2, -1),
    ((0, 0, 8), (0, 0, 1), True, (2.9, 3.1), 2, -1),
    ((0, 0, 15), (0, 0, -1), True, (1.9, 2.1), 2, 1),
    ((-5, 0, 5), (1, 0, 0), True, (3.9, 4.1), 0, -1),
    ((0, 0, 8), (0, 0, -1), True, (1.9, 2.1), 2, 1),
    ((3, 0, 0), (0, 0, 1), False, None, None, None),
    ((0, 10, 0), (0, 0, 1), False, None, None, None),
    ((0, 0, 0), (0, 0, -1), False, None, None, None),
    ((0, 0, 0), (0, 1, 0), True, (2.5, 3.5), 1, -1),
    ((3, 0, 0), (0, 1, 0), False, None, None, None),
    ((0, -5, 0), (0, 1, 0), True, (1.9, 2.2), 1, 1),
    ((25, 0, 0), (0, -1, 0), False, None, None, None),
]


def traverse_rays():
    r = np.zeros((len(TRAVERSE_RAYS), 8), np.float32)
    for i, (o, d, *_rest) in enumerate(TRAVERSE_RAYS):
        d = np.asarray(d, np.float32)
        r[i, 0:3] = o
        r[i, 4:7] = d / np.sqrt(np.float32(np.dot(d, d)))
        r[i, 7] = np.inf
    return r


def check_traverse_answers(hits_flag, t, n):
    for i, (_, _, want, trange, axis, sign) in enumerate(TRAVERSE_RAYS):
        assert bool(hits_flag[i]) == want, i
        if want:
            assert trange[0] <= t[i] <= trange[1], (i, t[i])
            assert np.sign(n[i, axis]) == sign, (i, n[i])


@needs_ref
def test_restatement_passes_test_traverse(orc):
    """The scene and the 12 rays of the reference's integration test, baked by the reference's
    sphere/box generators (its .scn reader), traced by the restatement."""
    ref = Reference("hybrid")
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "t.scn")
        open(p, "w").write(TEST_TRAVERSE_SCN)
        v, t = ref.scene_geometry(p)
    b = orc.build(v, t, make_cfg(**VARIANTS["hybrid"]))
    h, out, _, _, _ = orc.trace(b, traverse_rays())
    check_traverse_answers(h, out[:, 0], out[:, 3:6])
