"""The 8-wide traversal layout (rt_bvh_trace_loop form 2) against the oracle's restatement of
bvh::trace on the same baked tree.

Bar: every ray the reference hits is hit, with the closest distance bit-equal; the triangle
(and so u, v and the normal) may differ only where another triangle lies at exactly the same
distance (the visiting order decides such ties; scenes with coincident faces have many). A ray hit only through the conservative,
quantised child boxes -- a triangle that an exact box test loses by rounding at a box face --
is allowed, but must stay rare."""
import math

import numpy as np
import pytest

import rtb200
from oracle import Baked
from rtb200 import scenes
from test_gpu_build import SCENES
from test_gpu_trace import rays_for

pytestmark = pytest.mark.gpu


def _dec(p, q, s):
    """origin + q * 2^e in the float operations of the traversal's decode"""
    return np.float32(np.float32(p) + np.float32(np.float32(q) * np.float32(s)))


def _exponent(p, hi):
    ext = float(hi) - float(p)
    k = math.frexp(ext / 255.0)[1] if ext > 0 else 0
    e = min(max(k + 127, 1), 254)
    while e < 254 and _dec(p, 255, 2.0 ** (e - 127)) < hi:
        e += 1
    return e


def wide_restatement(nodes, scene_roots=()):
    """The wide layout restated on the host from the baked nodes (the rules of wide.cu)."""
    n = nodes.shape[0]
    leaf = nodes["is_leaf"].astype(bool)
    depth = np.zeros(n, np.int64)
    for i in range(n):  # pre-order: a parent precedes its children
        if not leaf[i]:
            depth[nodes["a"][i]] = depth[i] + 1
            depth[nodes["b"][i]] = depth[i] + 1
    flag = ~leaf & (depth % 3 == 0)
    for r in scene_roots:
        flag[r] |= not leaf[r]
    wid = np.cumsum(flag) - flag
    out = np.zeros(int(flag.sum()), rtb200.api.WIDE_NODE_DTYPE)
    for i in np.nonzero(flag)[0]:
        lst = [int(nodes["a"][i]), int(nodes["b"][i])]
        for _ in range(3):
            nl = []
            for c in lst:
                nl += [c] if (leaf[c] or flag[c]) else [int(nodes["a"][c]), int(nodes["b"][c])]
            lst = nl
        assert len(lst) <= 8
        pres = [not (leaf[c] and nodes["b"][c] == 0) and bool(np.all(nodes["bmin"][c][:3] <= nodes["bmax"][c][:3]))
                for c in lst]
        lo3 = [min(nodes["bmin"][c][a] for c, ok in zip(lst, pres) if ok) for a in range(3)]
        hi3 = [max(nodes["bmax"][c][a] for c, ok in zip(lst, pres) if ok) for a in range(3)]
        e = [_exponent(lo3[a], hi3[a]) for a in range(3)]
        # octant slots, greedily by the smallest cost (the first minimal pair wins)
        f32 = np.float32
        ctr = [f32(f32(f32(lo3[a]) + f32(hi3[a])) * f32(0.5)) for a in range(3)]
        off = {k: [f32(f32(f32(f32(nodes["bmin"][c][a]) + f32(nodes["bmax"][c][a])) * f32(0.5)) - ctr[a])
                   for a in range(3)] for k, (c, ok) in enumerate(zip(lst, pres)) if ok}
        slot, used = {}, set()
        for _ in range(len(off)):
            best = None
            for k in range(len(lst)):
                if k not in off or k in slot:
                    continue
                for sl in range(8):
                    if sl in used:
                        continue
                    o = off[k]
                    v = f32(f32((-o[0] if sl & 1 else o[0]) + (-o[1] if sl & 2 else o[1])) + (-o[2] if sl & 4 else o[2]))
                    if best is None or v < best[0]:
                        best = (v, k, sl)
            slot[best[1]] = best[2]
            used.add(best[2])
        w = out[wid[i]]
        w["p"] = lo3
        imask = 0
        for k0, (c, ok) in enumerate(zip(lst, pres)):
            if not ok:
                continue
            k = slot[k0]
            if leaf[c]:
                w["ref"][k], w["cnt"][k] = nodes["a"][c], nodes["b"][c]
            else:
                w["ref"][k], w["cnt"][k] = wid[c], 1
                imask |= 1 << k
            for a in range(3):
                s, p = 2.0 ** (e[a] - 127), lo3[a]
                lo = int(min(max(math.floor((float(nodes["bmin"][c][a]) - float(p)) / s), 0), 255))
                hi = int(min(max(math.ceil((float(nodes["bmax"][c][a]) - float(p)) / s), 0), 255))
                while lo > 0 and _dec(p, lo, s) > nodes["bmin"][c][a]:
                    lo -= 1
                while hi < 255 and _dec(p, hi, s) < nodes["bmax"][c][a]:
                    hi += 1
                assert _dec(p, lo, s) <= nodes["bmin"][c][a] and _dec(p, hi, s) >= nodes["bmax"][c][a]
                w["qlo"][a][k], w["qhi"][a][k] = lo, hi
        w["meta"] = e[0] | (e[1] << 8) | (e[2] << 16) | (imask << 24)
        out[wid[i]] = w
    return out


@pytest.mark.parametrize("scene,preset", [("soup20k", "hybrid"), ("soup20k", "lbvh63"), ("ico4", "sah4"),
                                          ("big_small", "hybrid"), ("identical100", "lbvh30")])
def test_wide_layout_matches_restatement(scene, preset):
    v, t = SCENES[scene]
    b = rtb200.Bvh.build(v, t, preset)
    b.trace_loop(2)
    got = b.wide_nodes()
    nodes = b.download()[0]
    exp = wide_restatement(nodes)
    assert got.shape == exp.shape
    if got.shape[0] == 0:  # a one-leaf tree: no wide nodes, the trace tests the leaf at once
        assert nodes["is_leaf"][0] == 1
        return
    for f in ("meta", "ref", "cnt", "qlo", "qhi", "pad"):
        bad = np.nonzero(np.any((got[f] != exp[f]).reshape(got.shape[0], -1), axis=1))[0]
        assert bad.size == 0, f"{scene}/{preset}: field {f} differs at wide nodes {bad[:8]}"
    assert np.array_equal(got["p"], exp["p"])  # value-equal (either zero)


def check_wide(hits, ref, tag, extra_frac=5e-4):
    h, out, tri, _, _ = ref
    g = (hits["flags"] & 1).astype(np.uint8)
    missed = np.nonzero((h == 1) & (g == 0))[0]
    assert missed.size == 0, f"{tag}: rays hit by the reference missed at {missed[:8]}"
    extra = np.nonzero((h == 0) & (g == 1))[0]
    assert extra.size <= extra_frac * h.size, f"{tag}: {extra.size} extra hits"
    m = (h == 1) & (g == 1)
    assert np.array_equal(hits["t"][m].view(np.uint32), out[m, 0].view(np.uint32)), f"{tag}: t differs"
    # a reported triangle is the one whose test produced the reported distance, so another
    # triangle with a bit-equal distance (checked above) is a tie at the closest distance
    diff = m & (hits["tri"] != tri)
    same = m & ~diff
    assert np.array_equal(hits["u"][same].view(np.uint32), out[same, 1].view(np.uint32)), f"{tag}: u differs"
    assert np.array_equal(hits["n"][same].view(np.uint32), out[same, 3:6].view(np.uint32)), f"{tag}: normals differ"
    return extra.size, int(diff.sum())


@pytest.mark.parametrize("preset", ["hybrid", "lbvh63", "lbvh30", "sah4"])
@pytest.mark.parametrize("scene", ["soup20k", "ico4", "cornell_ico", "big_small", "test_traverse", "identical100"])
def test_wide_matches_oracle(orc, scene, preset):
    v, t = SCENES[scene]
    b = rtb200.Bvh.build(v, t, preset)
    b.trace_loop(2)
    nodes, tris, verts = b.download()
    rays = rays_for(v, 40000, seed=17)
    hits = b.trace(rays)
    ref = orc.trace(Baked(nodes, tris, verts), rays, threads=8)
    check_wide(hits, ref, f"{scene}/{preset}")


def as_ref(hits):
    """binary-form hits in the oracle's tuple layout"""
    out = np.zeros((hits.shape[0], 6), np.float32)
    out[:, 0], out[:, 1], out[:, 2], out[:, 3:6] = hits["t"], hits["u"], hits["v"], hits["n"]
    return (hits["flags"] & 1).astype(np.uint8), out, hits["tri"], None, 0


@pytest.mark.parametrize("scene", ["soup20k", "cornell_ico", "big_small"])
def test_wide_watertight_matches_oracle(orc, scene):
    """The watertight mode in the wide form against the oracle's restatement of the watertight
    test (Woop, Benthin, Wald 2013; the reference has none) on the same tree, to the same bar."""
    v, t = SCENES[scene]
    b = rtb200.Bvh.build(v, t, "sah4")
    rays = rays_for(v, 40000, seed=21)
    ref = orc.trace(Baked(*b.download()), rays, flags=rtb200.TRACE_WATERTIGHT, threads=8)
    b.trace_loop(2)
    check_wide(b.trace(rays, rtb200.TRACE_WATERTIGHT), ref, f"{scene}/watertight")


def test_wide_any_hit_hits_the_same_rays(orc):
    """Any-hit returns the first accepted triangle of the visiting order: the same rays are hit,
    each with a triangle the ray really hits."""
    v, t = SCENES["soup20k"]
    b = rtb200.Bvh.build(v, t, "lbvh63")
    b.trace_loop(2)
    rays = rays_for(v, 40000, seed=18)
    closest = b.trace(rays, rtb200.TRACE_CLOSEST)
    anyh = b.trace(rays, rtb200.TRACE_ANY_HIT)
    assert np.array_equal(closest["flags"] & 1, anyh["flags"] & 1)
    m = (anyh["flags"] & 1) == 1
    assert np.all(anyh["t"][m] >= closest["t"][m])


def test_wide_follows_rebuilds_and_large_soup(orc):
    """The wide layout is rebuilt with the tree: a rebuild with another scene traces that scene;
    a 262,147-triangle soup exercises many wide levels."""
    b = rtb200.Bvh.build(*SCENES["soup2k"], "lbvh63")
    b.trace_loop(2)
    for v, t, preset in [(*SCENES["soup20k"], "sah4"), (*scenes.soup(262147, seed=77), "lbvh63")]:
        b.rebuild(v, t, preset)
        nodes, tris, verts = b.download()
        rays = rays_for(v, 60000, seed=19)
        ref = orc.trace(Baked(nodes, tris, verts), rays, threads=8)
        check_wide(b.trace(rays), ref, f"rebuild {preset}")
    b.trace_loop(-1)  # back to the reference's order: exact parity again
    ref = orc.trace(Baked(*b.download()), rays, threads=8)
    hits = b.trace(rays)
    h = ref[0] == 1
    assert np.array_equal((hits["flags"] & 1).astype(np.uint8), ref[0]) and np.array_equal(hits["tri"][h], ref[2][h])


def test_wide_batched_roots():
    """Scene roots of a batched build are wide nodes: the batched wavefront render (each scene's
    rays traced from its own root) matches the binary form's, up to the rare tie."""
    from test_gpu_batch import batch_setup, cfgs_for
    scs, bb, mats, mot = batch_setup(n=5)
    rcs = cfgs_for(scs, 48, 40, 4, max_bounce=4, rr_after=-1)
    img_bin, _ = bb.render_batch(rcs, mats, mot)
    bb.trace_loop(2)
    img_wide, _ = bb.render_batch(rcs, mats, mot)
    a, c = img_bin.cpu().numpy(), img_wide.cpu().numpy()
    assert np.mean(np.abs(a - c)) <= 1e-3 * max(float(np.mean(np.abs(a))), 1e-6)
    assert np.mean(np.isclose(a, c, rtol=1e-5, atol=1e-6)) > 0.999
