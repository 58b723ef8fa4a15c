"""Mesh ingestion on the host: the .scn `mesh <file> tx ty tz scale q qx qy qz qw` line
(src/bvh/bvh_IO.cpp:196-231) with the library's own PLY reader in place of the reference's
un-vendored importer (assimp with aiProcess_Triangulate | aiProcess_GenSmoothNormals,
bvh_IO.cpp:24-70).

Pinned: vertex and face counts, the polygon triangulation (a fan from each face's first corner),
index bounds and the error paths against an independent reader of the same files; the vertex
positions bit for bit against the reference's own transform code (translate * scale * toMat4,
the reference's math library, through oracle/_ref); and the bake of the reference's own
meshes (bunny.ply: 35,947 vertices with extra properties, 69,451 faces; letterX.ply: quads)
by the reference's bakeBVH against the oracle's restatement. Not pinned: the smooth normals a
mesh without normals receives -- the reference gets them from assimp, which is absent and which
no reference test exercises; the library accumulates area-weighted face normals and initGeos
renormalises them (bvh_IO.cpp:102-118)."""
import os
import tempfile

import numpy as np
import pytest

import rtb200
from mesh_files import fan, mixed_polygon_mesh, read_ply_raw, reference_mesh, write_ply
from oracle import Reference, VARIANTS, make_cfg

HAS_REF = Reference.available("hybrid")


def load_scn(text):
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "m.scn")
        open(p, "w").write(text)
        return rtb200.Mesh().read_scene(p).arrays()


TRANSFORMS = [((0.0, 0.0, 0.0), 1.0, (0.0, 0.0, 0.0, 1.0)),
              ((0.5, -1.25, 3.0), 2.5, (0.1, 0.7, -0.2, 0.68)),
              ((-3.0, 0.25, 1.0), 0.03, (0.0, 0.0, 0.3826834, 0.9238795))]


@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("with_normals", [False, True])
def test_ply_counts_triangulation_and_bounds(binary, with_normals):
    pos, faces = mixed_polygon_mesh()
    nrm = pos / np.linalg.norm(pos, axis=1, keepdims=True) if with_normals else None
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "m.ply")
        write_ply(p, pos, faces, normals=nrm, binary=binary)
        raw_pos, raw_faces = read_ply_raw(p)
        v, t = load_scn(f"mesh {p} 0 0 0 1 q 0 0 0 1\n")
    assert v.shape[0] == pos.shape[0] and t.shape[0] == sum(len(f) - 2 for f in faces)
    assert np.array_equal(t, fan(raw_faces))
    assert t.max() < v.shape[0]
    assert np.array_equal(v[:, :3], raw_pos)  # identity transform: positions unchanged
    n = np.linalg.norm(v[:, 3:], axis=1)
    assert np.all(n[np.unique(t)] > 0)  # vertices no face uses keep a zero normal (initGeos falls back to +Y)
    if with_normals:
        assert np.allclose(v[:, 3:], nrm, atol=1e-6)


def test_mesh_lines_append_with_offsets():
    pos, faces = mixed_polygon_mesh(seed=6)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "m.ply")
        write_ply(p, pos, faces, binary=True)
        v1, t1 = load_scn(f"mesh {p} 0 0 0 1 q 0 0 0 1\n")
        v2, t2 = load_scn(f"sphere 0 0 0 1\nmesh {p} 0 0 0 1 q 0 0 0 1\nmesh {p} 1 0 0 1 q 0 0 0 1\n")
    vs, ts = rtb200.Mesh().add_sphere((0.0, 0.0, 0.0), 1.0).arrays()
    assert v2.shape[0] == vs.shape[0] + 2 * v1.shape[0]
    assert np.array_equal(t2[ts.shape[0]:ts.shape[0] + t1.shape[0]], t1 + vs.shape[0])
    assert np.array_equal(t2[ts.shape[0] + t1.shape[0]:], t1 + vs.shape[0] + v1.shape[0])


@pytest.mark.skipif(not HAS_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("k", range(len(TRANSFORMS)))
def test_mesh_positions_match_reference_transform(k):
    """Positions bit for bit against loadMesh's transform in the reference's own math code;
    normals (when the file has them) to float rounding of the inverse-transpose."""
    tr, sc, (qx, qy, qz, qw) = TRANSFORMS[k]
    pos, faces = mixed_polygon_mesh(seed=7)
    nrm = pos / np.linalg.norm(pos, axis=1, keepdims=True)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "m.ply")
        write_ply(p, pos, faces, normals=nrm, binary=True)
        v, _ = load_scn(f"mesh {p} {tr[0]} {tr[1]} {tr[2]} {sc} q {qx} {qy} {qz} {qw}\n")
    want = Reference("hybrid").mesh_transform(tr, sc, (qw, qx, qy, qz), pos, nrm)
    assert np.array_equal(v[:, :3].view(np.uint32), want[:, :3].view(np.uint32))
    wn = want[:, 3:] / np.linalg.norm(want[:, 3:], axis=1, keepdims=True)
    gn = v[:, 3:] / np.linalg.norm(v[:, 3:], axis=1, keepdims=True)
    assert np.allclose(gn, wn, atol=2e-5)


def test_ply_errors():
    pos, faces = mixed_polygon_mesh(seed=8)
    with tempfile.TemporaryDirectory() as d:
        bad = os.path.join(d, "bad.ply")
        write_ply(bad, pos, faces[:-1] + [[0, 1, pos.shape[0] + 5]], binary=True)
        with pytest.raises(rtb200.RtError, match="RT_E_FORMAT"):
            load_scn(f"mesh {bad} 0 0 0 1 q 0 0 0 1\n")
        cut = os.path.join(d, "cut.ply")
        write_ply(cut, pos, faces, binary=True)
        data = open(cut, "rb").read()
        open(cut, "wb").write(data[: len(data) - 7])
        with pytest.raises(rtb200.RtError, match="RT_E_FORMAT"):
            load_scn(f"mesh {cut} 0 0 0 1 q 0 0 0 1\n")
        with pytest.raises(rtb200.RtError):
            load_scn(f"mesh {os.path.join(d, 'missing.ply')} 0 0 0 1 q 0 0 0 1\n")


@pytest.mark.skipif(reference_mesh("bunny.ply") is None, reason="reference meshes not copied (oracle/_ref)")
def test_reference_meshes_load():
    bunny = reference_mesh("bunny.ply")
    raw_pos, raw_faces = read_ply_raw(bunny)
    assert raw_pos.shape[0] == 35947 and len(raw_faces) == 69451
    v, t = load_scn(f"mesh {bunny} 0 0 0 1 q 0 0 0 1\n")
    assert v.shape[0] == 35947 and np.array_equal(t, fan(raw_faces))
    assert np.array_equal(v[:, :3], raw_pos)
    assert np.all(np.linalg.norm(v[:, 3:], axis=1)[np.unique(t)] > 0)
    for name, quads in (("letterX.ply", 2), ("letterY.ply", None)):
        path = reference_mesh(name)
        raw_pos, raw_faces = read_ply_raw(path)
        v, t = load_scn(f"mesh {path} 0 0 0 1 q 0 0 0 1\n")
        assert v.shape[0] == raw_pos.shape[0] and np.array_equal(t, fan(raw_faces)), name
        if quads is not None:
            assert len(raw_faces) == quads and all(len(f) == 4 for f in raw_faces) and t.shape[0] == 2 * quads


@pytest.mark.skipif(reference_mesh("bunny.ply") is None or not HAS_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("variant", ["hybrid", "lbvh63", "sah4"])
def test_reference_bakes_bunny_as_the_oracle_does(orc, variant):
    """The reference's own bakeBVH and the restatement give the same tree on the bunny, placed
    by a .scn mesh line with a rotation and scale."""
    bunny = reference_mesh("bunny.ply")
    v, t = load_scn(f"mesh {bunny} 0.2 -0.1 0.5 4.0 q 0.1 0.3 0.0 0.95\n")
    ref = Reference(variant).bake(v, t)
    res = orc.build(v, t, make_cfg(**VARIANTS[variant]))
    assert np.array_equal(ref.nodes[["is_leaf", "a", "b"]], res.nodes[["is_leaf", "a", "b"]])
    assert np.array_equal(ref.nodes["bmin"][:, :3], res.nodes["bmin"][:, :3])
    assert np.array_equal(ref.nodes["bmax"][:, :3], res.nodes["bmax"][:, :3])
    assert np.array_equal(ref.tris, res.tris)
    assert np.array_equal(ref.verts.view(np.uint32), res.verts.view(np.uint32))
