"""Pins the oracle's FP64 adjoint (orc_adjoint in oracle/rt_oracle.c) to its own forward path
loop before the GPU adjoint is checked against it: central finite differences of the
restated render (the same per-pixel Philox stream on both sides, so the two perturbed renders
follow the same paths) against the stored-path gradients, for per-triangle albedo and for the
light's emission. Runs on the CPU."""
import numpy as np

from oracle import OrcRenderCfg, make_cfg
from rtb200 import scenes


def baked_to_orig(baked_tris, tris):
    """original triangle index of each baked triangle (vertex triples are unique here)"""
    idx = {tuple(r): i for i, r in enumerate(tris.tolist())}
    return np.array([idx[tuple(r)] for r in baked_tris.tolist()], np.int64)


def small_diff_case(orc, rr_after=-1):
    cv, ct, cid = scenes.cornell()
    iv, it = scenes.icosphere(1, center=(0.0, -0.4, 0.2), radius=0.45, seed=21)
    v, t, part = scenes.concat([(cv, ct), (iv, it)])
    obj = np.concatenate([cid, np.full(it.shape[0], 6, np.uint32)])
    mats = [dict(albedo=(0.75, 0.75, 0.75)), dict(albedo=(0.75, 0.75, 0.75)), dict(albedo=(0.75, 0.75, 0.75)),
            dict(albedo=(0.65, 0.1, 0.1)), dict(albedo=(0.1, 0.6, 0.15)),
            dict(albedo=(0.0, 0.0, 0.0), emission=(15.0, 15.0, 15.0)), dict(albedo=(0.5, 0.5, 0.5))]
    baked = orc.build(v, t, make_cfg(lbvh_threshold=0, morton_bits=10))
    orig = baked_to_orig(baked.tris, t)
    mot = obj[orig].astype(np.uint32)
    rng = np.random.default_rng(5)
    talb = rng.uniform(0.2, 0.8, size=(t.shape[0], 3)).astype(np.float32)[orig]
    rc = OrcRenderCfg()
    rc.width, rc.height, rc.spp, rc.max_bounce, rc.rr_after, rc.env_kind = 14, 12, 4, 3, rr_after, 1
    rc.env_color[:] = [0.0, 0.0, 0.0]
    rc.cam_pos[:] = [0.0, 0.0, -2.9]; rc.cam_fwd[:] = [0.0, 0.0, 1.0]
    rc.cam_right[:] = [1.0, 0.0, 0.0]; rc.cam_up[:] = [0.0, 1.0, 0.0]
    rc.tan_half_fov_y = float(np.tan(np.radians(22.5)))
    rc.seed, rc.sample_offset = 9, 0
    d = rng.uniform(0.5, 1.5, size=(rc.height, rc.width, 3)).astype(np.float32)
    return baked, mats, mot, talb, rc, d


def loss(orc, baked, rc, mats, mot, talb, d):
    img, _ = orc.render(baked, rc, mats, mot, tri_albedo=talb, threads=4)
    return float(np.sum(d.astype(np.float64) * img.astype(np.float64)))


def test_oracle_adjoint_matches_finite_differences(orc):
    baked, mats, mot, talb, rc, d = small_diff_case(orc)
    g_alb, g_em = orc.adjoint(baked, rc, d, mats, mot, talb, threads=4)
    assert np.abs(g_alb).max() > 0 and np.abs(g_em[5]).max() > 0
    h = 1e-2
    flat = np.argsort(-np.abs(g_alb).ravel())[:12]
    for k in flat:
        tri, c = divmod(int(k), 3)
        tp, tm = talb.copy(), talb.copy()
        tp[tri, c] += h; tm[tri, c] -= h
        fd = (loss(orc, baked, rc, mats, mot, tp, d) - loss(orc, baked, rc, mats, mot, tm, d)) / (2 * h)
        assert abs(fd - g_alb[tri, c]) <= 1e-2 * abs(fd) + 1e-6, (tri, c, fd, g_alb[tri, c])
    for c in range(3):
        mp = [dict(m) for m in mats]; mm = [dict(m) for m in mats]
        e = list(mats[5]["emission"]); e[c] += h; mp[5]["emission"] = tuple(e)
        e = list(mats[5]["emission"]); e[c] -= h; mm[5]["emission"] = tuple(e)
        fd = (loss(orc, baked, rc, mp, mot, talb, d) - loss(orc, baked, rc, mm, mot, talb, d)) / (2 * h)
        assert abs(fd - g_em[5, c]) <= 1e-2 * abs(fd) + 1e-6, (c, fd, g_em[5, c])


def test_oracle_adjoint_zero_weights_give_zero_gradients(orc):
    baked, mats, mot, talb, rc, d = small_diff_case(orc)
    g_alb, g_em = orc.adjoint(baked, rc, np.zeros_like(d), mats, mot, talb, threads=2)
    assert not g_alb.any() and not g_em.any()


def test_oracle_adjoint_is_linear_in_the_weights(orc):
    baked, mats, mot, talb, rc, d = small_diff_case(orc, rr_after=1)
    g1, e1 = orc.adjoint(baked, rc, d, mats, mot, talb, threads=3)
    g2, e2 = orc.adjoint(baked, rc, 2.0 * d, mats, mot, talb, threads=1)
    assert np.allclose(g2, 2.0 * g1, rtol=1e-12, atol=1e-15)
    assert np.allclose(e2, 2.0 * e1, rtol=1e-12, atol=1e-15)
