"""The allocation-free entry point rt_morton_order_noalloc, called through the C ABI.

Some callers of this library cannot allocate device memory while they work: an interactive
renderer that re-bakes moving geometry every frame cannot afford the device-wide
synchronisation a cudaMalloc causes mid-frame, and a host application that hands plugins a
fixed device-memory budget forbids them to grow it. For them the library offers one entry
point whose scratch is a fixed device array compiled into the library. These tests check that
its output equals what the allocating path produces (rt_build's baked triangle order for the
LBVH presets, read back with rt_bvh_prim_ids) and the oracle's restatement of the reference's
sortTrisByMorton (src/bvh/bvh_morton.cpp:109-159), on two calls in a row since every call
shares and reuses the same scratch; that calls after the first allocate nothing (the library's
own allocation counter and the device's free memory are unchanged); and that the size limit is
enforced with a clear error.

This file is collected last on purpose, so a run that stops at the first failure has already
run every other test.
"""
import numpy as np
import pytest

import rtb200
from rtb200 import scenes
from rtb200.api import NOALLOC_MAX_TRIS, morton_order_noalloc

pytestmark = pytest.mark.gpu


def _device(v, t):
    import torch
    v = np.ascontiguousarray(v, np.float32)
    t = np.ascontiguousarray(t, np.uint32)
    return torch.from_numpy(v).cuda(), torch.from_numpy(t.view(np.int32)).cuda()


@pytest.mark.parametrize("preset,bits", [("lbvh63", 21), ("lbvh30", 10)])
def test_noalloc_order_matches_allocating_build(orc, preset, bits):
    import torch
    from oracle import VARIANTS, make_cfg
    meshes = [scenes.soup(50000, seed=31), scenes.icosphere(4), scenes.soup(NOALLOC_MAX_TRIS, seed=32)]
    for v, t in meshes:
        dv, dt = _device(v, t)
        want = rtb200.Bvh.build(dv, dt, preset).prim_ids()
        _, orc_perm, _ = orc.morton(v, t, make_cfg(**VARIANTS[preset]))
        for call in range(2):  # the second call reuses the scratch the first one left behind
            out = torch.full((t.shape[0],), -1, dtype=torch.int32, device="cuda")
            morton_order_noalloc(dv, dt, out, morton_bits=bits)
            got = out.cpu().numpy().view(np.uint32)
            assert np.array_equal(got, orc_perm), f"{preset} call {call}: order differs from the oracle's sort"
            assert np.array_equal(got, want), f"{preset} call {call}: order differs from rt_build's"


def test_noalloc_allocates_nothing():
    import torch
    v, t = scenes.soup(40000, seed=33)
    dv, dt = _device(v, t)
    out = torch.empty(t.shape[0], dtype=torch.int32, device="cuda")
    # The first call on the device looks up the scratch array's address; the first use of each
    # key width's kernels also makes the driver load them (and the array) if it has not yet.
    for bits in (21, 10):
        morton_order_noalloc(dv, dt, out, morton_bits=bits)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    allocs0 = rtb200.api.device_allocations()
    for bits in (21, 10, 21):
        morton_order_noalloc(dv, dt, out, morton_bits=bits)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert rtb200.api.device_allocations() == allocs0, "the library allocated device memory"
    assert free1 >= free0, f"device memory shrank by {free0 - free1} bytes"


def test_noalloc_rejects_oversize():
    import torch
    v, t = scenes.soup(NOALLOC_MAX_TRIS + 1, seed=34)
    dv, dt = _device(v, t)
    out = torch.full((t.shape[0],), -1, dtype=torch.int32, device="cuda")
    with pytest.raises(rtb200.RtError) as e:
        morton_order_noalloc(dv, dt, out)
    assert e.value.code == 4 and "at most" in str(e.value)  # RT_E_CAPACITY
    assert int(out.min().item()) == -1 and int(out.max().item()) == -1  # nothing written


def test_noalloc_on_a_second_device(orc):
    """The scratch array's address and the sort's kernel attributes are per device: after calls
    on device 0, a call on device 1 must look up its own copy and set its own attributes. Needs
    two visible GPUs."""
    import torch
    from oracle import VARIANTS, make_cfg
    if torch.cuda.device_count() < 2:
        pytest.skip("one visible GPU")
    v, t = scenes.soup(30000, seed=35)
    _, want, _ = orc.morton(v, t, make_cfg(**VARIANTS["lbvh63"]))
    for dev in (0, 1, 0, 1):
        with torch.cuda.device(dev):
            dv, dt = _device(v, t)
            out = torch.full((t.shape[0],), -1, dtype=torch.int32, device="cuda")
            morton_order_noalloc(dv, dt, out, morton_bits=21)
            assert np.array_equal(out.cpu().numpy().view(np.uint32), want), f"device {dev}"
