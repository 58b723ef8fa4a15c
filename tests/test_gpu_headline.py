"""Parity at the BVH microbenchmark's own sizes: the seeded 1,048,576-triangle soup that bench.py
bakes (scenes.soup(1 << 20, seed=BASE_SEED + 1)), its 16,777,216 incoherent rays and its
1920 x 1080 pinhole primary rays.

* Trees: the GPU's bake against the oracle's restatement of bvh::bakeBVH
  (src/bvh/bvh_bake.cpp:180-194) node for node, for the LBVH presets with 63- and 30-bit codes,
  the reference's default hybrid and the binned SAH with spatial splits and leaf 4.
* Traversal: bvh::trace (src/bvh/bvh_traverse.cpp:237-246) restated, on the GPU's trees (equal
  to the oracle's by the tree tests): the first 1,048,576 of the 16,777,216 incoherent rays the
  GPU traced in one call, and all 2,073,600 primary rays; closest and any hit. Bar: identical
  hit flags and triangles, t / u / v and normals bit-equal."""
import os

import numpy as np
import pytest

import rtb200
from oracle import Baked
from rtb200 import scenes
from test_gpu_build import assert_same_tree, orc_cfg
from test_gpu_trace import compare

pytestmark = pytest.mark.gpu

N_TRIS = 1 << 20
N_INCOHERENT = 1 << 24
SLICE = 1 << 20
THREADS = os.cpu_count() or 1
_SOUP = {}


def soup():
    if not _SOUP:
        _SOUP["vt"] = scenes.soup(N_TRIS, seed=scenes.BASE_SEED + 1)
    return _SOUP["vt"]


@pytest.mark.parametrize("preset", ["lbvh63", "lbvh30", "hybrid", "sah4"])
def test_headline_soup_tree_matches_oracle(orc, preset):
    v, t = soup()
    b = rtb200.Bvh.build(v, t, preset)
    ref = orc.build(v, t, orc_cfg(preset))
    assert_same_tree(b.download(), ref, f"1M soup/{preset}")
    assert np.array_equal(t[b.prim_ids()], ref.tris)
    st = b.stats()
    assert st["spatial_taken"] == int(ref.stats[0]) and st["spatial_refused"] == int(ref.stats[1])


@pytest.mark.parametrize("flags", [rtb200.TRACE_CLOSEST, rtb200.TRACE_ANY_HIT])
@pytest.mark.parametrize("preset", ["lbvh63", "sah4"])
def test_headline_rays_match_oracle(orc, preset, flags):
    import torch
    v, t = soup()
    b = rtb200.Bvh.build(v, t, preset)
    baked = Baked(*b.download())
    lo, hi = v[:, :3].min(0), v[:, :3].max(0)
    rays = scenes.incoherent_rays(N_INCOHERENT, lo, hi, seed=scenes.BASE_SEED + 9)
    d_hits = b.trace(torch.from_numpy(rays).cuda(), flags)
    hits = d_hits[:SLICE].cpu().numpy().view(rtb200.HIT_DTYPE).reshape(-1)
    del d_hits
    compare(hits, orc.trace(baked, rays[:SLICE], flags=flags, threads=THREADS), f"{preset}/incoherent/{flags}")
    del rays
    prim = scenes.pinhole_rays(1920, 1080, (0.5, 0.5, -1.5), (0.5, 0.5, 0.5), 60.0)
    hits = b.trace(prim, flags)
    compare(hits, orc.trace(baked, prim, flags=flags, threads=THREADS), f"{preset}/primary1080p/{flags}")
