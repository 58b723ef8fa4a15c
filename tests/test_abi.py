"""C-ABI surface and host-side logic of librt_b200.so, on the CPU (no compute calls):

* the library loads and exports every function include/rt_b200.h declares;
* the host geometry (the reference's sphere / box generators and its .scn grammar) is bit-equal
  to the reference's own readScene (oracle/_ref);
* .bvh v1 error paths of loadBVH (src/bvh/bvh_traverse.cpp:185-230) are reported as codes;
* without a CUDA device the compute entry points fail loudly (no CPU fallback).
"""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

import rtb200
from conftest import has_cuda
from oracle import Reference
from rtb200 import api
from scenes_for_tests import TEST_TRAVERSE_SCN


def test_exports_every_declared_symbol():
    L = rtb200.lib()
    declared = rtb200.header_symbols()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert L.rt_version().startswith(b"rt_b200")


def test_default_cfg_is_the_reference_constants():
    c = rtb200.make_cfg("hybrid")
    assert (c.lbvh_threshold, c.max_leaf, c.morton_bits, c.bins_min, c.bins_max) == (64, 16, 21, 8, 32)
    assert abs(c.c_trav - 1.0) < 1e-7 and abs(c.c_isect - 1.2) < 1e-7 and abs(c.spatial_mult - 1.5) < 1e-7


SCN = TEST_TRAVERSE_SCN + (
    "sphere 1 2 3 0.5 8 12\n"
    "box 1 1 1 0.5 0.25 2 q 0.1 0.2 0.3 0.9273618\n"
    "box 0 0 0 1 1 1 z 0 0 0 1\n"        # unknown orientation type: identity (bvh_IO.cpp:175-179)
    "sphere 0, 0, 0, 1000\n"             # malformed: skipped (as testscene.scn's line is)
    "# a comment\nbrdf 1 2 3\n")


@pytest.mark.skipif(not Reference.available("hybrid"), reason="oracle/_ref not built")
def test_scene_geometry_matches_reference():
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "s.scn")
        open(p, "w").write(SCN)
        v, t = rtb200.Mesh().read_scene(p).arrays()
        rv, rt = Reference("hybrid").scene_geometry(p)
    assert v.shape == rv.shape and np.array_equal(v.view(np.uint32), rv.view(np.uint32))
    assert np.array_equal(t, rt)


def test_sphere_and_box_counts():
    """Counts pinned by the reference's tests/test_geo.cpp: 2+(r-1)s vertices, 2s(r-1) triangles;
    24 vertices / 12 triangles per box."""
    m = rtb200.Mesh().add_sphere((0, 0, 0), 1.0, 6, 10)
    v, t = m.arrays()
    assert v.shape[0] == 2 + 5 * 10 and t.shape[0] == 2 * 10 * 5
    assert np.allclose(np.linalg.norm(v[:, :3], axis=1), 1.0, atol=1e-6)
    m.add_box((3, 0, 0), (1, 2, 3))
    v2, t2 = m.arrays()
    assert v2.shape[0] - v.shape[0] == 24 and t2.shape[0] - t.shape[0] == 12
    assert t2[t.shape[0]:].min() >= v.shape[0]  # appended (bvh_geo.cpp appends to the shared arrays)


def _write(path, header, payload=b""):
    with open(path, "wb") as f:
        f.write(np.array(header, "<u4").tobytes())
        f.write(payload)


def test_bvh_file_errors_are_codes():
    L = rtb200.lib()
    out = C.c_void_p()
    with tempfile.TemporaryDirectory() as d:
        assert L.rt_load_bvh(os.path.join(d, "missing.bvh").encode(), C.byref(out)) == 2  # RT_E_IO
        p = os.path.join(d, "v2.bvh")
        _write(p, [2, 1, 0, 0], bytes(48))
        assert L.rt_load_bvh(p.encode(), C.byref(out)) == 3  # version mismatch: RT_E_FORMAT
        p = os.path.join(d, "short.bvh")
        _write(p, [1, 5, 3, 9], bytes(100))
        assert L.rt_load_bvh(p.encode(), C.byref(out)) == 3  # truncated payload
        with open(os.path.join(d, "hdr.bvh"), "wb") as f:
            f.write(b"\x01\x00")
        assert L.rt_load_bvh(os.path.join(d, "hdr.bvh").encode(), C.byref(out)) == 3  # truncated header
    assert not out.value


def test_bvh_structure_is_checked_before_upload():
    L = rtb200.lib()
    nodes = np.zeros(3, api.NODE_DTYPE)
    nodes[0]["is_leaf"], nodes[0]["a"], nodes[0]["b"] = 0, 1, 7  # child beyond the array
    nodes[1]["is_leaf"], nodes[1]["a"], nodes[1]["b"] = 1, 0, 1
    tris = np.zeros((1, 3), np.uint32)
    verts = np.zeros((3, 6), np.float32)
    out = C.c_void_p()
    code = L.rt_bvh_from_arrays(nodes.ctypes.data_as(C.c_void_p), 3, tris.ctypes.data_as(C.c_void_p), 1,
                                verts.ctypes.data_as(C.c_void_p), 3, C.byref(out))
    assert code in (3, 6)  # RT_E_FORMAT (or RT_E_CUDA first on a machine without a device)


@pytest.mark.skipif(has_cuda(), reason="checks the behaviour without a CUDA device")
def test_no_cpu_fallback_without_a_device():
    v = np.zeros((3, 6), np.float32)
    v[1, 0] = 1.0
    v[2, 1] = 1.0
    t = np.array([[0, 1, 2]], np.uint32)
    with pytest.raises(rtb200.RtError) as e:
        rtb200.Bvh.build(v, t)
    assert e.value.code == 6 and "CUDA" in str(e.value)
