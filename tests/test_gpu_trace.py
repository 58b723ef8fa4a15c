"""GPU traversal parity: librt_b200's trace against the oracle's restatement of bvh::trace on
the same baked BVH. Bar: identical hit flags and triangle indices, t/u/v and normals bit-equal."""
import numpy as np
import pytest

import rtb200
from oracle import Baked
from rtb200 import scenes
from scenes_for_tests import scene_set
from test_gpu_build import SCENES

pytestmark = pytest.mark.gpu


def rays_for(v, n, seed):
    lo, hi = v[:, :3].min(0), v[:, :3].max(0)
    pad = 0.1 * (hi - lo) + 1e-3
    r = scenes.incoherent_rays(n, lo - pad, hi + pad, seed=seed)
    # axis-parallel rays through box planes: the NaN slabs of rayAABB
    k = n // 8
    r[:k, 4:7] = 0.0
    r[np.arange(k), 4 + np.arange(k) % 3] = np.where(np.arange(k) % 2, 1.0, -1.0)
    r[: k // 2, 0] = v[np.arange(k // 2) % v.shape[0], 0]
    return r


def compare(hits, ref, tag):
    h, out, tri, _, _ = ref
    gh = (hits["flags"] & 1).astype(np.uint8)
    assert np.array_equal(gh, h), f"{tag}: hit flags differ at {np.nonzero(gh != h)[0][:8]}"
    m = h == 1
    assert np.array_equal(hits["tri"][m], tri[m]), f"{tag}: triangle ids differ"
    assert np.array_equal(hits["t"][m].view(np.uint32), out[m, 0].view(np.uint32)), f"{tag}: t differs"
    assert np.array_equal(hits["u"][m].view(np.uint32), out[m, 1].view(np.uint32)), f"{tag}: u differs"
    assert np.array_equal(hits["v"][m].view(np.uint32), out[m, 2].view(np.uint32)), f"{tag}: v differs"
    assert np.array_equal(hits["n"][m].view(np.uint32), out[m, 3:6].view(np.uint32)), f"{tag}: normals differ"


@pytest.mark.parametrize("preset", ["hybrid", "lbvh30", "sah4"])
@pytest.mark.parametrize("scene", ["soup20k", "ico4", "cornell_ico", "big_small", "test_traverse", "identical100"])
@pytest.mark.parametrize("flags", [rtb200.TRACE_CLOSEST, rtb200.TRACE_ANY_HIT, rtb200.TRACE_WATERTIGHT,
                                   rtb200.TRACE_WATERTIGHT | rtb200.TRACE_ANY_HIT])
@pytest.mark.parametrize("loop", [0, 1])
def test_trace_matches_oracle(orc, scene, preset, flags, loop):
    """Both traversal loop forms (one-loop, while-while) against the oracle: the any-hit mode
    returns the first accepted triangle, so it checks the visiting order itself. The watertight
    modes against the oracle's own restatement of Woop, Benthin and Wald (2013)."""
    v, t = SCENES[scene]
    b = rtb200.Bvh.build(v, t, preset)
    b.trace_loop(loop)
    nodes, tris, verts = b.download()
    rays = rays_for(v, 40000, seed=7)
    hits = b.trace(rays, flags)
    ref = orc.trace(Baked(nodes, tris, verts), rays, flags=flags, threads=8)
    compare(hits, ref, f"{scene}/{preset}/{flags}/loop{loop}")


def test_trace_device_tensors(orc):
    import torch
    v, t = SCENES["soup20k"]
    b = rtb200.Bvh.build(v, t, "hybrid")
    rays = rays_for(v, 100000, seed=9)
    dh = b.trace(torch.from_numpy(rays).cuda())
    hits = dh.cpu().numpy().view(rtb200.HIT_DTYPE).reshape(-1)
    nodes, tris, verts = b.download()
    compare(hits, orc.trace(Baked(nodes, tris, verts), rays, threads=8), "device")
