"""The reference's own tests, compiled unchanged against this repository's drop-in headers and
librt_b200.so (oracle/build_ref.sh builds them from the reference tree into oracle/_ref/tests):
tests/test_aabb.cpp (host AABB helpers, CPU) and tests/test_traverse.cpp (bakeBVH -> loadBVH ->
trace of 12 rays, on the GPU)."""
import os
import subprocess
import tempfile

import pytest

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "tests")


def _run(name):
    exe = os.path.join(BIN, name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (oracle/build_ref.sh needs the reference tree)")
    with tempfile.TemporaryDirectory() as d:  # test_traverse writes its scene and .bvh in the cwd
        p = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=300)
    return p.returncode, p.stdout + p.stderr


def test_reference_test_aabb_passes():
    rc, out = _run("test_aabb")
    assert rc == 0, out[-2000:]
    assert "Results: 106/106 passed" in out


@pytest.mark.gpu
def test_reference_test_traverse_passes():
    rc, out = _run("test_traverse")
    assert rc == 0, out[-3000:]
    assert "Results: 27/27 passed" in out
