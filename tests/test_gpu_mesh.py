"""GPU bake and traversal of meshes that came in through a .scn `mesh` line (PLY files: the
reference's own bunny.ply when it was copied next to the reference build, and a seeded mesh of
triangles, quads and pentagons written here): the tree node for node and the hits triangle for
triangle against the oracle's restatement on the same loaded geometry, and the .bvh file that
rt_bake_scene writes for the scene against the same tree."""
import os
import tempfile

import numpy as np
import pytest

import rtb200
from mesh_files import mixed_polygon_mesh, reference_mesh, write_ply
from oracle import Baked
from test_gpu_build import assert_same_tree, orc_cfg
from test_gpu_trace import compare, rays_for

pytestmark = pytest.mark.gpu


def mesh_scene(d, which):
    if which == "bunny":
        path = reference_mesh("bunny.ply")
        if path is None:
            pytest.skip("reference meshes not copied (oracle/_ref)")
        line = f"mesh {path} 0.2 -0.1 0.5 4.0 q 0.1 0.3 0.0 0.95\n"
    else:
        pos, faces = mixed_polygon_mesh(seed=9)
        path = os.path.join(d, "mixed.ply")
        write_ply(path, pos, faces, binary=True)
        line = f"mesh {path} 1.0 2.0 -0.5 0.75 q 0.0 0.38268343 0.0 0.9238795\n"
    scn = os.path.join(d, "m.scn")
    open(scn, "w").write(line + "sphere 0 0 3 0.5\n")
    return scn


@pytest.mark.parametrize("preset", ["hybrid", "lbvh63", "sah4"])
@pytest.mark.parametrize("which", ["bunny", "mixed"])
def test_mesh_bake_and_trace_match_oracle(orc, which, preset):
    with tempfile.TemporaryDirectory() as d:
        scn = mesh_scene(d, which)
        v, t = rtb200.Mesh().read_scene(scn).arrays()
        b = rtb200.Bvh.build(v, t, preset)
        ref = orc.build(v, t, orc_cfg(preset))
        assert_same_tree(b.download(), ref, f"{which}/{preset}")
        rays = rays_for(v, 40000, seed=13)
        for flags in (rtb200.TRACE_CLOSEST, rtb200.TRACE_ANY_HIT):
            compare(b.trace(rays, flags), orc.trace(ref, rays, flags=flags, threads=8), f"{which}/{preset}/{flags}")
        if preset == "hybrid":  # bvh::bakeBVH's own entry: .scn in, .bvh out
            out = os.path.join(d, "m.bvh")
            rtb200.bake_scene(scn, out)
            f = Baked.read_bvh(out)
            assert_same_tree((f.nodes, f.tris, f.verts), ref, f"{which}/bake_scene")
