"""GPU bake parity: librt_b200's build against the C restatement oracle (itself pinned bit for
bit against the reference in test_oracle.py), for every build preset on seeded scenes.

Bar: identical tree -- node kinds, child / triangle indices and triangle order equal, boxes
value-equal (+0 and -0 compare equal: the reference's own choice between them depends on the
order it extends boxes in), vertices bit-equal (normals renormalised as initGeos does)."""
import os
import tempfile

import numpy as np
import pytest

import rtb200
from oracle import make_cfg as orc_make_cfg
from rtb200 import scenes
from scenes_for_tests import scene_set

pytestmark = pytest.mark.gpu

PRESETS = ["hybrid", "lbvh63", "lbvh30", "lbvh63l4", "sah4", "sah16", "sah4ns"]


def read_scn(text):
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "s.scn")
        open(p, "w").write(text)
        return rtb200.Mesh().read_scene(p).arrays()


SCENES = scene_set(read_scn)


def orc_cfg(preset):
    kw = dict(rtb200.PRESETS[preset])
    if kw["lbvh_threshold"] == 0xFFFFFFFF:
        kw["lbvh_threshold"] = 0xFFFFFFFF
    return orc_make_cfg(**kw)


def assert_same_tree(gpu, ref, tag):
    gn, gt, gv = gpu
    assert gn.shape == ref.nodes.shape, f"{tag}: node count {gn.shape[0]} vs {ref.nodes.shape[0]}"
    for f in ("is_leaf", "a", "b"):
        bad = np.nonzero(gn[f] != ref.nodes[f])[0]
        assert bad.size == 0, f"{tag}: field {f} differs at nodes {bad[:8]}"
    for f in ("bmin", "bmax"):
        bad = np.nonzero(np.any(gn[f] != ref.nodes[f], axis=1))[0]
        assert bad.size == 0, f"{tag}: {f} differs at nodes {bad[:8]}: {gn[f][bad[:2]]} vs {ref.nodes[f][bad[:2]]}"
    assert np.array_equal(gt, ref.tris), f"{tag}: triangle order differs"
    assert np.array_equal(gv.view(np.uint32), ref.verts.view(np.uint32)), f"{tag}: vertices differ"


@pytest.mark.parametrize("preset", PRESETS)
@pytest.mark.parametrize("scene", sorted(SCENES))
def test_build_matches_oracle(orc, scene, preset):
    v, t = SCENES[scene]
    ref = orc.build(v, t, orc_cfg(preset))
    b = rtb200.Bvh.build(v, t, preset)
    assert_same_tree(b.download(), ref, f"{scene}/{preset}")
    # original triangle ids of the baked order
    pid = b.prim_ids()
    assert np.array_equal(t[pid], ref.tris)
    st = b.stats()
    assert st["spatial_taken"] == int(ref.stats[0]) and st["spatial_refused"] == int(ref.stats[1])


def test_build_from_device_tensors(orc):
    import torch
    v, t = SCENES["soup20k"]
    ref = orc.build(v, t, orc_cfg("hybrid"))
    dv = torch.from_numpy(v).cuda()
    dt = torch.from_numpy(t.view(np.int32)).cuda()
    b = rtb200.Bvh.build(dv, dt, "hybrid")
    assert_same_tree(b.download(), ref, "device-in")


def test_rebuild_reuses_handle(orc):
    b = rtb200.Bvh.build(*SCENES["soup2k"], "lbvh63")
    for name in ("soup20k", "ico4", "soup2k"):
        v, t = SCENES[name]
        b.rebuild(v, t, "lbvh63")
        assert_same_tree(b.download(), orc.build(v, t, orc_cfg("lbvh63")), f"rebuild {name}")


def test_rebuild_replays_with_new_contents(orc):
    """Bakes of one size from the same device buffers replay a captured launch graph from the
    third bake on; new contents in those buffers give the new tree every time."""
    import torch
    (v1, t1), (v2, t2) = scenes.soup(20000, seed=91), scenes.soup(20000, seed=92)
    dv = torch.from_numpy(v1).cuda()
    dt = torch.from_numpy(t1.view(np.int32)).cuda()
    b = rtb200.Bvh.build(dv, dt, "lbvh63")
    for k in range(5):
        v, t = (v1, t1) if k % 2 == 0 else (v2, t2)
        dv.copy_(torch.from_numpy(v))
        dt.copy_(torch.from_numpy(t.view(np.int32)))
        torch.cuda.synchronize()
        b.rebuild(dv, dt, "lbvh63")
        assert_same_tree(b.download(), orc.build(v, t, orc_cfg("lbvh63")), f"bake {k}")
        assert np.array_equal(t[b.prim_ids()], b.download()[1])


@pytest.mark.parametrize("preset", ["lbvh63", "lbvh30"])
def test_replayed_bake_sorts_clustered_keys(orc, preset):
    """A replayed bake leaves the sort's LSD fallback out; when new contents put more keys in a
    top-digit bucket than one block sorts, the kernels after the sort return at once (their
    inputs are not sorted) and the bake is done again launch by launch, so the tree is still
    the oracle's. The clustered contents come first too: the first replay of a handle (the
    second bake) can be the one that overflows."""
    import torch
    n = 200_000
    vu, tu = scenes.soup(n, seed=93)
    vc, tc = clustered_soup(n, seed=94)
    dv = torch.from_numpy(vc).cuda()
    dt = torch.from_numpy(tc.view(np.int32)).cuda()
    b = rtb200.Bvh.build(dv, dt, preset)
    for k, (v, t) in enumerate([(vc, tc), (vc, tc), (vu, tu), (vu, tu), (vc, tc), (vu, tu), (vc, tc)]):
        dv.copy_(torch.from_numpy(v))
        dt.copy_(torch.from_numpy(t.view(np.int32)))
        torch.cuda.synchronize()
        b.rebuild(dv, dt, preset)
        assert_same_tree(b.download(), orc.build(v, t, orc_cfg(preset)), f"bake {k}")


def test_errors_are_reported():
    v, t = SCENES["soup2k"]
    bad = t.copy()
    bad[5, 1] = v.shape[0] + 7
    with pytest.raises(rtb200.RtError) as e:
        rtb200.Bvh.build(v, bad)
    assert e.value.code == 9  # RT_E_INDEX, the reference's initGeos index check
    with pytest.raises(rtb200.RtError) as e:
        rtb200.Bvh.build(v[:0], t[:0])
    assert e.value.code == 8  # RT_E_EMPTY


@pytest.mark.parametrize("preset", ["lbvh63", "lbvh30", "hybrid", "sah4", "sah16"])
def test_large_odd_soup_matches_oracle(orc, preset):
    """262,147 triangles: 1,025 tiles of the local tree phase (the last one partial), frontier
    nodes on every tile edge; for the SAH presets the top levels' nodes above 16,384
    references, which many blocks evaluate at once."""
    v, t = scenes.soup(262147, seed=77)
    ref = orc.build(v, t, orc_cfg(preset))
    b = rtb200.Bvh.build(v, t, preset)
    assert_same_tree(b.download(), ref, f"soup262147/{preset}")
    st = b.stats()
    assert st["spatial_taken"] == int(ref.stats[0]) and st["spatial_refused"] == int(ref.stats[1])


def test_sort_tile_shapes_agree(orc):
    """2^21 + 5 triangles run the 8-keys-per-thread sort; its Morton order is the oracle's."""
    v, t = scenes.soup((1 << 21) + 5, seed=78)
    codes, perm, _ = orc.morton(v, t, orc_cfg("lbvh63"))
    b = rtb200.Bvh.build(v, t, "lbvh63l4")
    pid = b.prim_ids()
    # leaves of the LBVH presets hold sorted runs: the baked order is the stable Morton order
    assert np.array_equal(pid, perm)


def clustered_soup(n, seed):
    """90% of the triangles inside 5% of the box: the top Morton digit's first bucket holds far
    more than one block's worth of keys."""
    v, t = scenes.soup(n, seed=seed)
    v = v.copy()
    v[: 3 * (9 * n // 10), :3] *= 0.05
    return v, t


@pytest.mark.parametrize("case", ["uniform1m", "uniform1500k", "uniform3k", "clustered200k"])
@pytest.mark.parametrize("preset", ["lbvh63", "lbvh30"])
def test_sort_msd_and_lsd_paths_agree(orc, case, preset):
    """Uniform soups take the sort's MSD + per-bucket path (every top-digit bucket fits one
    block: 4,608-key blocks up to about 1.09M keys, 8,192-key blocks above), the clustered one
    its LSD passes; all give the oracle's stable Morton order."""
    if case == "uniform1m":
        v, t = scenes.soup(1_000_003, seed=81)
    elif case == "uniform1500k":
        v, t = scenes.soup(1_500_001, seed=84)
    elif case == "uniform3k":
        v, t = scenes.soup(3001, seed=82)
    else:
        v, t = clustered_soup(200_000, seed=83)
    codes, perm, _ = orc.morton(v, t, orc_cfg(preset))
    if case == "clustered200k":
        top = np.asarray(codes, np.uint64) >> np.uint64(55 if preset == "lbvh63" else 22)  # bits key_bits-8 ..
        assert np.bincount(top.astype(np.int64)).max() > 8192
    pid = rtb200.Bvh.build(v, t, preset).prim_ids()
    assert np.array_equal(pid, perm)


def test_download_async_on_a_stream(orc):
    """rt_bvh_download_async: the .bvh arrays land in pinned host memory once the stream has
    reached the copies, equal to the synchronous download."""
    import ctypes as C
    import torch
    v, t = SCENES["soup20k"]
    b = rtb200.Bvh.build(v, t, "lbvh63")
    nn, nt, nv = b.counts()
    s = torch.cuda.Stream()
    hn = torch.empty(nn * 48, dtype=torch.uint8).pin_memory()
    ht = torch.empty(nt * 12, dtype=torch.uint8).pin_memory()
    hv = torch.empty(nv * 24, dtype=torch.uint8).pin_memory()
    assert rtb200.lib().rt_bvh_download_async(b.h, C.c_void_p(hn.data_ptr()), C.c_void_p(ht.data_ptr()),
                                              C.c_void_p(hv.data_ptr()), C.c_void_p(s.cuda_stream)) == 0
    s.synchronize()
    nodes, tris, verts = b.download()
    assert np.array_equal(hn.numpy(), nodes.view(np.uint8))
    assert np.array_equal(ht.numpy(), tris.view(np.uint8).reshape(-1))
    assert np.array_equal(hv.numpy(), verts.view(np.uint8).reshape(-1))


def test_build_on_every_visible_device(orc):
    """Kernel attributes (the sort's and the climb's shared-memory limits above 48 KB) are
    per-device settings: a bake on device 1 after device 0 in the same process must launch with
    them set there too. Needs two visible GPUs."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("one visible GPU")
    v, t = scenes.soup(300000, seed=41)  # MSD sort path with 63-bit keys, climb with its shared-memory tiles
    ref = orc.build(v, t, orc_cfg("lbvh63"))
    for dev in range(torch.cuda.device_count()):
        with torch.cuda.device(dev):
            b = rtb200.Bvh.build(torch.from_numpy(v).cuda(), torch.from_numpy(t.view(np.int32)).cuda(), "lbvh63")
            assert_same_tree(b.download(), ref, f"device {dev}")
