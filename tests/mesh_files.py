"""PLY writing and reading for the mesh-ingestion tests: a writer for seeded test meshes (ASCII
or binary little-endian, optional normals, extra per-vertex properties, n-gon faces) and an
independent reader of the raw element data, both plain numpy, to check the library's loader
(the .scn `mesh` line, src/bvh/bvh_IO.cpp:196-231, whose importer the reference does not
vendor) against."""
import os

import numpy as np

from oracle import REF_MESH_DIR


def write_ply(path, pos, faces, normals=None, extra=("confidence", "intensity"), binary=False, seed=0):
    """pos: (V, 3); faces: list of index lists (any length >= 3); extra: names of additional
    float vertex properties (filled with seeded values) placed after the position."""
    rng = np.random.default_rng(seed)
    pos = np.asarray(pos, np.float32)
    cols = [pos]
    names = ["x", "y", "z"]
    if normals is not None:
        cols.append(np.asarray(normals, np.float32))
        names += ["nx", "ny", "nz"]
    for e in extra:
        cols.append(rng.random((pos.shape[0], 1), dtype=np.float32))
        names.append(e)
    vdata = np.concatenate(cols, axis=1).astype(np.float32)
    hdr = ["ply", f"format {'binary_little_endian' if binary else 'ascii'} 1.0", "comment seeded test mesh",
           f"element vertex {pos.shape[0]}"]
    hdr += [f"property float {n}" for n in names]
    hdr += [f"element face {len(faces)}", "property list uchar int vertex_indices", "end_header"]
    with open(path, "wb") as f:
        f.write(("\n".join(hdr) + "\n").encode())
        if binary:
            f.write(vdata.astype("<f4").tobytes())
            for fc in faces:
                f.write(np.uint8(len(fc)).tobytes())
                f.write(np.asarray(fc, "<i4").tobytes())
        else:
            for row in vdata:
                f.write((" ".join(repr(float(x)) for x in row) + "\n").encode())
            for fc in faces:
                f.write((" ".join(str(int(x)) for x in [len(fc)] + list(fc)) + "\n").encode())


def read_ply_raw(path):
    """(positions (V, 3) float32, faces as a list of index lists) of an ASCII or binary
    little-endian PLY with a float x / y / z vertex and a face list element."""
    with open(path, "rb") as f:
        data = f.read()
    end = data.index(b"end_header") + len(b"end_header")
    end = data.index(b"\n", end) + 1
    header = data[:end].decode().splitlines()
    binary = any(l.startswith("format binary_little_endian") for l in header)
    elems = []
    for l in header:
        w = l.split()
        if not w:
            continue
        if w[0] == "element":
            elems.append([w[1], int(w[2]), []])
        elif w[0] == "property":
            elems[-1][2].append(w[1:])
    sizes = {"char": 1, "uchar": 1, "int8": 1, "uint8": 1, "short": 2, "ushort": 2, "int16": 2, "uint16": 2,
             "int": 4, "uint": 4, "int32": 4, "uint32": 4, "float": 4, "float32": 4, "double": 8, "float64": 8}
    kinds = {"char": "i1", "uchar": "u1", "int8": "i1", "uint8": "u1", "short": "<i2", "ushort": "<u2", "int16": "<i2",
             "uint16": "<u2", "int": "<i4", "uint": "<u4", "int32": "<i4", "uint32": "<u4", "float": "<f4",
             "float32": "<f4", "double": "<f8", "float64": "<f8"}
    pos, faces = None, []
    if binary:
        off = end
        for name, count, props in elems:
            if all(p[0] != "list" for p in props):
                dt = np.dtype([(p[1], kinds[p[0]]) for p in props])
                arr = np.frombuffer(data, dt, count, off)
                off += dt.itemsize * count
                if name == "vertex":
                    pos = np.stack([arr["x"], arr["y"], arr["z"]], 1).astype(np.float32)
            else:
                for _ in range(count):
                    for p in props:
                        if p[0] == "list":
                            n = int(np.frombuffer(data, kinds[p[1]], 1, off)[0]); off += sizes[p[1]]
                            items = np.frombuffer(data, kinds[p[2]], n, off).astype(np.int64); off += sizes[p[2]] * n
                            if name == "face":
                                faces.append(list(items))
                        else:
                            off += sizes[p[0]]
    else:
        toks = data[end:].split()
        k = 0
        for name, count, props in elems:
            rows = []
            for _ in range(count):
                row = {}
                for p in props:
                    if p[0] == "list":
                        n = int(toks[k]); k += 1
                        row[p[-1]] = [int(x) for x in toks[k:k + n]]; k += n
                    else:
                        row[p[1]] = float(toks[k]); k += 1
                rows.append(row)
            if name == "vertex":
                pos = np.array([[r["x"], r["y"], r["z"]] for r in rows], np.float32)
            elif name == "face":
                faces = [next(v for key, v in r.items() if isinstance(v, list)) for r in rows]
    return pos, faces


def fan(faces):
    """Triangles of a face list by fanning each polygon from its first corner."""
    return np.array([[fc[0], fc[j], fc[j + 1]] for fc in faces for j in range(1, len(fc) - 1)], np.uint32)


def reference_mesh(name):
    """Path of one of the reference's own mesh files copied next to its build, or None."""
    p = os.path.join(REF_MESH_DIR, name)
    return p if os.path.exists(p) else None


def mixed_polygon_mesh(seed=5):
    """A seeded closed-ish mesh with mixed polygons: an icosphere's triangles, plus quads and
    pentagons built on a second ring of vertices."""
    from rtb200 import scenes
    v, t = scenes.icosphere(3, center=(0.0, 0.0, 0.0), radius=1.0, seed=seed)
    pos = v[:, :3].copy()
    faces = [list(map(int, f)) for f in t]
    rng = np.random.default_rng(seed)
    ring = rng.uniform(-1.5, 1.5, size=(40, 3)).astype(np.float32)
    base = pos.shape[0]
    pos = np.concatenate([pos, ring])
    for i in range(0, 36, 4):
        faces.append([base + i, base + i + 1, base + i + 2, base + i + 3])
    for i in range(0, 35, 5):
        faces.append([base + i, base + i + 1, base + i + 2, base + i + 3, base + i + 4])
    return pos, faces
