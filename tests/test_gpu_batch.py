"""Batched scenes: rt_build_batch against rt_build of every scene alone (bit-identical
subtrees, triangles and vertices after renumbering), rt_render_batch against a render of every
scene alone with the same camera and seed (the same samples; the wavefront's atomic
accumulation order is the only difference), the CUDA-graph replay, and the autotuner."""
import numpy as np
import pytest
import torch

import rtb200
from rtb200 import scenes

pytestmark = pytest.mark.gpu


def same_arrays(a, b, tag):
    (na, ta, va), (nb, tb, vb) = a, b
    assert na.shape == nb.shape, (tag, na.shape, nb.shape)
    for f in ("is_leaf", "a", "b"):
        assert np.array_equal(na[f], nb[f]), (tag, f)
    for f in ("bmin", "bmax"):
        assert np.array_equal(na[f][:, :3].view(np.uint32), nb[f][:, :3].view(np.uint32)), (tag, f)
    assert np.array_equal(ta, tb), tag
    assert np.array_equal(va.view(np.uint32), vb.view(np.uint32)), tag


def mixed_parts(seed=0):
    parts = [scenes.soup(1500, seed=seed + 1), scenes.icosphere(3, seed=seed + 2), scenes.soup(1, seed=seed + 3),
             scenes.soup(7, seed=seed + 4), scenes.icosphere(4, center=(2.0, 0.0, 0.0), seed=seed + 5),
             scenes.soup(20000, seed=seed + 6), scenes.soup(17, seed=seed + 7)]
    return parts


@pytest.mark.parametrize("preset,kw", [("lbvh30", {}), ("lbvh30", dict(max_leaf=4)),
                                       ("hybrid", dict(morton_bits=10)), ("sah4", dict(morton_bits=10))])
def test_batched_build_matches_single_builds(preset, kw):
    parts = mixed_parts()
    cfg = rtb200.make_cfg(preset, **kw)
    v, t, vo, to = rtb200.batch_arrays(parts)
    bb = rtb200.Bvh.build_batch(v, t, vo, to, cfg)
    info = bb.scenes()
    assert info.shape == (len(parts), 4)
    dl = bb.download()
    for s, (pv, pt) in enumerate(parts):
        single = rtb200.Bvh.build(pv, pt, cfg)
        same_arrays(bb.scene_arrays(s, vo, dl), single.download(), f"{preset} scene {s}")


def test_batched_build_device_input_and_many_scenes():
    parts = [scenes.soup(int(n), seed=100 + i) for i, n in enumerate(np.geomspace(1, 3000, 64).astype(int))]
    v, t, vo, to = rtb200.batch_arrays(parts)
    bb = rtb200.Bvh.build_batch(torch.from_numpy(v).cuda(), torch.from_numpy(t.view(np.int32)).cuda(), vo, to, "lbvh30")
    dl = bb.download()
    for s in (0, 1, 17, 40, 63):
        single = rtb200.Bvh.build(*parts[s], "lbvh30")
        same_arrays(bb.scene_arrays(s, vo, dl), single.download(), f"scene {s}")
    # a rebuild of another batch into the same handle
    parts2 = parts[10:20]
    v2, t2, vo2, to2 = rtb200.batch_arrays(parts2)
    bb.rebuild_batch(v2, t2, vo2, to2, "lbvh30")
    dl = bb.download()
    assert bb.scenes().shape == (10, 4)
    for s in (0, 9):
        same_arrays(bb.scene_arrays(s, vo2, dl), rtb200.Bvh.build(*parts2[s], "lbvh30").download(), f"rebuild {s}")


def test_batched_build_errors():
    parts = mixed_parts()[:3]
    v, t, vo, to = rtb200.batch_arrays(parts)
    with pytest.raises(rtb200.RtError, match="RT_E_INVALID"):
        rtb200.Bvh.build_batch(v, t, vo, to, "lbvh63")          # 63 + 2 key bits
    bad = to.copy(); bad[2] = bad[1]
    with pytest.raises(rtb200.RtError, match="RT_E_EMPTY"):
        rtb200.Bvh.build_batch(v, t, vo, bad, "lbvh30")
    tt = t.copy(); tt[to[1]] = [0, 1, vo[2] - vo[1]]            # index past scene 1's vertices
    with pytest.raises(rtb200.RtError, match="RT_E_INDEX"):
        rtb200.Bvh.build_batch(v, tt, vo, to, "lbvh30")
    two = rtb200.Bvh.build_batch(*rtb200.batch_arrays(parts[:2]), "lbvh63")  # 63 + 1 bits fit
    assert two.scenes().shape == (2, 4)


def batch_setup(n=6, lo=500, hi=20000, seed=5):
    scs = scenes.batch_scenes(n, lo, hi, seed=seed)
    v, t, vo, to = rtb200.batch_arrays([(sc.verts, sc.tris) for sc in scs])
    bb = rtb200.Bvh.build_batch(v, t, vo, to, "lbvh30")
    mats, mot_in = scenes.batch_shading(scs)
    mot = mot_in[bb.prim_ids()]
    return scs, bb, mats, mot


def cfgs_for(scs, w, h, spp, **kw):
    return [rtb200.render_cfg(w, h, spp, lookat=sc.lookat, env_kind=1, seed=31 + i, **kw) for i, sc in enumerate(scs)]


@pytest.mark.parametrize("rr_after", [-1, 2])
def test_batched_render_matches_single_scene_renders(rr_after):
    scs, bb, mats, mot = batch_setup()
    rcs = cfgs_for(scs, 48, 40, 8, max_bounce=5, rr_after=rr_after)
    img, img2 = bb.render_batch(rcs, mats, mot, want_sq=True)
    for s, sc in enumerate(scs):
        single = rtb200.Bvh.build(sc.verts, sc.tris, "lbvh30")
        ref, ref2 = single.render(rcs[s], sc.mats, sc.baked_materials(single.prim_ids()), mode=rtb200.RENDER_PLAIN,
                                  want_sq=True)
        assert np.allclose(img[s].cpu().numpy(), ref.cpu().numpy(), rtol=1e-5, atol=1e-6), s
        assert np.allclose(img2[s].cpu().numpy(), ref2.cpu().numpy(), rtol=1e-5, atol=1e-5), s


def test_graph_replay_and_autotune():
    scs, bb, mats, mot = batch_setup(n=4)
    rcs = cfgs_for(scs, 64, 48, 4, max_bounce=4, rr_after=-1)
    a, _ = bb.render_batch(rcs, mats, mot)
    b, _ = bb.render_batch(rcs, mats, mot)                     # replays the captured graph
    assert np.allclose(a.cpu().numpy(), b.cpu().numpy(), rtol=1e-5, atol=1e-6)
    depth = bb.depth()
    assert 0 < depth < 64
    best = bb.autotune(rcs, mats, mot)
    d = best.as_dict()
    assert d["trace_block"] in (64, 128, 256) and d["chunk_paths"] in (1 << 20, 1 << 21, 1 << 22, 1 << 23)
    assert d["stack_depth"] in (32, 64) and (d["stack_depth"] == 64 or depth + 1 <= 32)
    c, _ = bb.render_batch(rcs, mats, mot)                     # the tuned parameters
    assert np.allclose(a.cpu().numpy(), c.cpu().numpy(), rtol=1e-5, atol=1e-6)
    small = rtb200.WavefrontParams(64, 4096, 64, 128)          # many chunks
    e, _ = bb.render_batch(rcs, mats, mot, params=small)
    assert np.allclose(a.cpu().numpy(), e.cpu().numpy(), rtol=1e-5, atol=1e-6)
    with pytest.raises(rtb200.RtError, match="RT_E_INVALID"):
        bb.render_batch(rcs[:2], mats, mot)
