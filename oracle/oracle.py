"""ctypes front end of the test oracles (TEST INFRASTRUCTURE ONLY).

Two checkers live here:

* ``Restatement`` -- liboracle.so, the plain-C restatement of the reference algorithm
  (oracle/rt_oracle.c), which runs anywhere (it is what travels with the tests);
* ``Reference`` -- oracle/_ref/<variant>/libref.so, the reference's own BVH sources
  compiled in place by oracle/build_ref.sh, present where the reference tree was.

Only tests/, the smoke check and bench.py's CPU-baseline leg import this module, and only
to check or time against the product; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "lib", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
# the reference's own mesh files, copied next to its build by oracle/build_ref.sh
REF_MESH_DIR = os.path.join(REF_DIR, "meshes")

# Build parameter sets: the reference's compile-time constants of each oracle/_ref variant
# (oracle/build_ref.sh) as runtime values.
VARIANTS = {
    "hybrid":   dict(lbvh_threshold=64, max_leaf=16, morton_bits=21),
    "lbvh63":   dict(lbvh_threshold=0, max_leaf=16, morton_bits=21),
    "lbvh30":   dict(lbvh_threshold=0, max_leaf=16, morton_bits=10),
    "lbvh63l4": dict(lbvh_threshold=0, max_leaf=4, morton_bits=21),
    "sah4":     dict(lbvh_threshold=2147483647, max_leaf=4, morton_bits=21),
    "sah16":    dict(lbvh_threshold=2147483647, max_leaf=16, morton_bits=21),
    "sah4ns":   dict(lbvh_threshold=2147483647, max_leaf=4, morton_bits=21, spatial_eps=3.0e38),
}

NODE_DTYPE = np.dtype([("bmin", "<f4", 4), ("bmax", "<f4", 4), ("is_leaf", "u1"), ("pad0", "u1", 3),
                       ("a", "<u4"), ("b", "<u4"), ("pad1", "<u4")])
assert NODE_DTYPE.itemsize == 48


class OrcCfg(C.Structure):
    _fields_ = [("lbvh_threshold", C.c_uint32), ("max_leaf", C.c_uint32), ("morton_bits", C.c_uint32),
                ("bins_min", C.c_uint32), ("bins_max", C.c_uint32), ("c_trav", C.c_float),
                ("c_isect", C.c_float), ("centroid_eps", C.c_float), ("spatial_eps", C.c_float),
                ("spatial_mult", C.c_float)]


class OrcMaterial(C.Structure):
    _fields_ = [("albedo", C.c_float * 3), ("emission", C.c_float * 3), ("kind", C.c_uint32),
                ("pad", C.c_uint32)]


class OrcRenderCfg(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32),
                ("max_bounce", C.c_uint32), ("rr_after", C.c_int32), ("env_kind", C.c_uint32),
                ("env_color", C.c_float * 3), ("cam_pos", C.c_float * 3), ("cam_fwd", C.c_float * 3),
                ("cam_right", C.c_float * 3), ("cam_up", C.c_float * 3), ("tan_half_fov_y", C.c_float),
                ("seed", C.c_uint32), ("sample_offset", C.c_uint32)]


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def make_cfg(**kw) -> OrcCfg:
    c = OrcCfg(64, 16, 21, 8, 32, 1.0, 1.2, 1e-6, 1e-6, 1.5)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


class Baked:
    """A baked BVH in the .bvh v1 layout: nodes (48-byte records), triangles, vertices."""

    def __init__(self, nodes, tris, verts, stats=None):
        self.nodes, self.tris, self.verts, self.stats = nodes, tris, verts, stats

    @staticmethod
    def read_bvh(path) -> "Baked":
        """Reads a .bvh v1 file (src/bvh/bvh_IO.cpp:236-275 writes it)."""
        raw = np.fromfile(path, dtype=np.uint8)
        hdr = raw[:16].view("<u4")
        ver, nn, nt, nv = (int(x) for x in hdr)
        assert ver == 1, ver
        o = 16
        nodes = raw[o:o + 48 * nn].view(NODE_DTYPE).copy(); o += 48 * nn
        tris = raw[o:o + 12 * nt].view("<u4").reshape(nt, 3).copy(); o += 12 * nt
        verts = raw[o:o + 24 * nv].view("<f4").reshape(nv, 6).copy(); o += 24 * nv
        assert o == raw.size
        return Baked(nodes, tris, verts)


class Restatement:
    """liboracle.so: the C restatement (oracle/rt_oracle.c)."""

    def __init__(self, path: str = ORACLE_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = C.CDLL(path)
        self.L = L
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        L.orc_morton.argtypes = [vp, u32, vp, u32, vp, vp, vp, vp]
        L.orc_build.restype = vp
        L.orc_build.argtypes = [vp, u32, vp, u32, vp]
        L.orc_counts.argtypes = [vp, vp]
        L.orc_stats.argtypes = [vp, vp]
        L.orc_get.argtypes = [vp, vp, vp, vp]
        L.orc_free.argtypes = [vp]
        L.orc_from_arrays.restype = vp
        L.orc_from_arrays.argtypes = [vp, u32, vp, u32, vp, u32]
        L.orc_normalize_normals.argtypes = [vp, u32]
        L.orc_clip_triangle.argtypes = [vp, vp, vp]
        L.orc_trace.restype = u64
        L.orc_trace.argtypes = [vp, vp, u64, u32, vp, vp, vp, vp, C.c_int]
        L.orc_render.argtypes = [vp, vp, vp, vp, u32, u32, vp, vp, C.c_int]
        L.orc_render_ex.argtypes = [vp, vp, vp, u32, vp, vp, vp, u32, u32, u32, u32, vp, vp, C.c_int]
        L.orc_adjoint.argtypes = [vp, vp, vp, u32, vp, vp, vp, vp, vp, C.c_int]
        L.orc_philox.argtypes = [u32, u32, u32, u32, u32, u32, vp]
        L.orc_primary_rays.argtypes = [vp, u64, vp, vp, vp, vp, vp]
        L.orc_render_stats.argtypes = [vp, vp, vp, u32, vp, vp, vp, u32, u32, u32, u32, vp, vp, C.c_int]
        L.orc_trace_brute.argtypes = [vp, vp, u32, vp, u64, u32, vp, vp, vp]
        L.orc_cosine_dirs.argtypes = [u64, vp, vp, vp, vp]
        L.orc_ibl_lookup.argtypes = [vp, u32, u32, u64, vp, vp]

    def morton(self, verts, tris, cfg: OrcCfg):
        verts = np.ascontiguousarray(verts, np.float32); tris = np.ascontiguousarray(tris, np.uint32)
        n = tris.shape[0]
        codes = np.zeros(n, np.uint64); perm = np.zeros(n, np.uint32); sb = np.zeros(6, np.float32)
        ok = self.L.orc_morton(_p(verts), verts.shape[0], _p(tris), n, C.byref(cfg), _p(codes), _p(perm), _p(sb))
        assert ok
        return codes, perm, sb

    def build(self, verts, tris, cfg: OrcCfg) -> Baked | None:
        verts = np.ascontiguousarray(verts, np.float32); tris = np.ascontiguousarray(tris, np.uint32)
        h = self.L.orc_build(_p(verts), verts.shape[0], _p(tris), tris.shape[0], C.byref(cfg))
        if not h:
            return None
        cnt = np.zeros(3, np.uint32); st = np.zeros(4, np.uint32)
        self.L.orc_counts(h, _p(cnt)); self.L.orc_stats(h, _p(st))
        nodes = np.zeros(int(cnt[0]), NODE_DTYPE)
        ot = np.zeros((int(cnt[1]), 3), np.uint32)
        ov = np.zeros((int(cnt[2]), 6), np.float32)
        self.L.orc_get(h, _p(nodes), _p(ot), _p(ov))
        self.L.orc_free(h)
        return Baked(nodes, ot, ov, st)

    def normalize_normals(self, verts):
        v = np.ascontiguousarray(verts, np.float32).copy()
        self.L.orc_normalize_normals(_p(v), v.shape[0])
        return v

    def clip_triangle(self, v9, box6):
        v9 = np.ascontiguousarray(v9, np.float32); box6 = np.ascontiguousarray(box6, np.float32)
        out = np.zeros(6, np.float32)
        self.L.orc_clip_triangle(_p(v9), _p(box6), _p(out))
        return out

    def trace(self, baked: Baked, rays, flags: int = 0, threads: int = 1, counters: bool = False):
        """rays: (n, 8) float32 = o.xyz, tmin, d.xyz, tmax. Returns hit, t/u/v/n, tri, counters, overflow."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        h = self.L.orc_from_arrays(_p(baked.nodes), baked.nodes.shape[0], _p(baked.tris), baked.tris.shape[0],
                                   _p(baked.verts), baked.verts.shape[0])
        out = np.zeros((n, 6), np.float32); tri = np.zeros(n, np.uint32); hit = np.zeros(n, np.uint8)
        ctr = np.zeros((n, 3), np.uint32) if counters else None
        of = self.L.orc_trace(h, _p(rays), n, flags, _p(out), _p(tri), _p(hit), _p(ctr), threads)
        self.L.orc_free(h)
        return hit, out, tri, ctr, int(of)

    @staticmethod
    def _mats(mats, mat_of_tri):
        if mats is None:
            return None, None
        arr = (OrcMaterial * len(mats))()
        for i, m in enumerate(mats):
            arr[i].albedo[:] = list(m["albedo"]); arr[i].emission[:] = list(m.get("emission", (0, 0, 0)))
            arr[i].kind = int(m.get("kind", 0))
        mot = np.ascontiguousarray(mat_of_tri, np.uint32) if mat_of_tri is not None else None
        return arr, mot

    def _handle(self, baked: Baked):
        return self.L.orc_from_arrays(_p(baked.nodes), baked.nodes.shape[0], _p(baked.tris), baked.tris.shape[0],
                                      _p(baked.verts), baked.verts.shape[0])

    def render(self, baked: Baked, rcfg: OrcRenderCfg, mats=None, mat_of_tri=None, rows=None, threads: int = 1,
               want_sq: bool = False, tri_albedo=None, env_map=None):
        """Image rows [r0, r1) of the path loop; tri_albedo: (n_tris, 3) albedo per baked triangle;
        env_map: (h, w, 3) equirectangular map for env_kind 2."""
        W, H = rcfg.width, rcfg.height
        rgb = np.zeros((H, W, 3), np.float32)
        rgb2 = np.zeros((H, W, 3), np.float32) if want_sq else None
        hnd = self._handle(baked)
        r0, r1 = rows if rows is not None else (0, H)
        mats_arr, mot = self._mats(mats, mat_of_tri)
        ta = np.ascontiguousarray(tri_albedo, np.float32) if tri_albedo is not None else None
        em = np.ascontiguousarray(env_map, np.float32) if env_map is not None else None
        eh, ew = (em.shape[0], em.shape[1]) if em is not None else (0, 0)
        self.L.orc_render_ex(hnd, C.byref(rcfg), mats_arr, len(mats) if mats is not None else 0, _p(mot), _p(ta),
                             _p(em), ew, eh, r0, r1, _p(rgb), _p(rgb2), threads)
        self.L.orc_free(hnd)
        return rgb, rgb2

    def render_stats(self, baked: Baked, rcfg: OrcRenderCfg, mats=None, mat_of_tri=None, rows=None, threads: int = 1,
                     tri_albedo=None, env_map=None):
        """Rows [r0, r1) of render() plus its traversal work: (rgb, (segments traced, nodes
        popped, triangles tested) summed over every sample of those rows)."""
        W, H = rcfg.width, rcfg.height
        rgb = np.zeros((H, W, 3), np.float32)
        hnd = self._handle(baked)
        r0, r1 = rows if rows is not None else (0, H)
        mats_arr, mot = self._mats(mats, mat_of_tri)
        ta = np.ascontiguousarray(tri_albedo, np.float32) if tri_albedo is not None else None
        em = np.ascontiguousarray(env_map, np.float32) if env_map is not None else None
        eh, ew = (em.shape[0], em.shape[1]) if em is not None else (0, 0)
        counts = np.zeros(3, np.uint64)
        self.L.orc_render_stats(hnd, C.byref(rcfg), mats_arr, len(mats) if mats is not None else 0, _p(mot), _p(ta),
                                _p(em), ew, eh, r0, r1, _p(rgb), _p(counts), threads)
        self.L.orc_free(hnd)
        return rgb, tuple(int(x) for x in counts)

    def adjoint(self, baked: Baked, rcfg: OrcRenderCfg, d_rgb, mats=None, mat_of_tri=None, tri_albedo=None,
                threads: int = 1):
        """FP64 gradients (n_tris, 3) and (n_mats, 3) of sum(d_rgb * image)."""
        hnd = self._handle(baked)
        mats_arr, mot = self._mats(mats, mat_of_tri)
        ta = np.ascontiguousarray(tri_albedo, np.float32) if tri_albedo is not None else None
        d = np.ascontiguousarray(d_rgb, np.float32)
        g_alb = np.zeros((baked.tris.shape[0], 3), np.float64)
        g_em = np.zeros((len(mats), 3), np.float64) if mats is not None else None
        self.L.orc_adjoint(hnd, C.byref(rcfg), mats_arr, len(mats) if mats is not None else 0, _p(mot), _p(ta), _p(d),
                           _p(g_alb), _p(g_em), threads)
        self.L.orc_free(hnd)
        return g_alb, g_em

    def trace_brute(self, verts, tris, rays, flags: int = 0):
        """Every ray against every triangle (no BVH): hit, (n, 3) t / u / v, triangle."""
        verts = np.ascontiguousarray(verts, np.float32); tris = np.ascontiguousarray(tris, np.uint32)
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        out = np.zeros((n, 3), np.float32); tri = np.zeros(n, np.uint32); hit = np.zeros(n, np.uint8)
        self.L.orc_trace_brute(_p(verts), _p(tris), tris.shape[0], _p(rays), n, flags, _p(out), _p(tri), _p(hit))
        return hit, out, tri

    def primary_rays(self, rcfg: OrcRenderCfg, px, py, jx, jy):
        px = np.ascontiguousarray(px, np.int32); py = np.ascontiguousarray(py, np.int32)
        jx = np.ascontiguousarray(jx, np.float32); jy = np.ascontiguousarray(jy, np.float32)
        out = np.zeros((px.shape[0], 8), np.float32)
        self.L.orc_primary_rays(C.byref(rcfg), px.shape[0], _p(px), _p(py), _p(jx), _p(jy), _p(out))
        return out

    def cosine_dirs(self, u1, u2, normals):
        u1 = np.ascontiguousarray(u1, np.float32); u2 = np.ascontiguousarray(u2, np.float32)
        nrm = np.ascontiguousarray(normals, np.float32)
        out = np.zeros((u1.shape[0], 3), np.float32)
        self.L.orc_cosine_dirs(u1.shape[0], _p(u1), _p(u2), _p(nrm), _p(out))
        return out

    def ibl_lookup(self, env_map, dirs):
        em = np.ascontiguousarray(env_map, np.float32); d = np.ascontiguousarray(dirs, np.float32)
        out = np.zeros((d.shape[0], 3), np.float32)
        self.L.orc_ibl_lookup(_p(em), em.shape[1], em.shape[0], d.shape[0], _p(d), _p(out))
        return out

    def philox(self, c, k):
        out = np.zeros(4, np.uint32)
        self.L.orc_philox(*[int(x) for x in c], *[int(x) for x in k], _p(out))
        return out


class Reference:
    """oracle/_ref/<variant>/libref.so: the reference's own bake/load/trace."""

    def __init__(self, variant: str = "hybrid"):
        path = os.path.join(REF_DIR, variant, "libref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        self.L = L
        self.variant = variant
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        L.ref_constants.argtypes = [vp]
        L.ref_bake_arrays.argtypes = [vp, u32, vp, u32, C.c_char_p]
        L.ref_bake_scene.argtypes = [C.c_char_p]
        L.ref_scene_geometry.argtypes = [C.c_char_p, vp, vp, vp]
        L.ref_morton.argtypes = [vp, u32, vp, u32, vp, vp, vp]
        L.ref_init_geos.argtypes = [vp, u32, vp, u32]
        L.ref_load.argtypes = [C.c_char_p]
        L.ref_trace.argtypes = [vp, u64, vp, vp, vp, C.c_int]
        L.ref_clip_triangle.argtypes = [vp, vp, vp]
        L.ref_mesh_transform.argtypes = [vp, C.c_float, vp, u64, vp, vp, vp]
        # the path loop of src/main.cpp (oracle/ref_main_harness.cpp)
        i32 = C.c_int
        L.ref_scene_config.argtypes = [C.c_char_p, vp, vp, vp]
        L.ref_camera_lookat.argtypes = [vp, vp, C.c_float, vp]
        L.ref_camera_quat.argtypes = [vp, vp, C.c_float, vp]
        L.ref_primary_rays.argtypes = [vp, i32, i32, u64, vp, vp, vp, vp, vp]
        L.ref_cosine_dirs.argtypes = [u64, vp, vp, vp, vp]
        L.ref_ibl_lookup.argtypes = [vp, i32, i32, u64, vp, vp]
        L.ref_path_render.argtypes = [vp, i32, i32, i32, i32, u32, vp, i32, i32, i32, i32, vp, vp, i32]

    @staticmethod
    def available(variant: str = "hybrid") -> bool:
        return os.path.exists(os.path.join(REF_DIR, variant, "libref.so"))

    def constants(self):
        out = np.zeros(6, np.int32)
        self.L.ref_constants(_p(out))
        return out

    def bake(self, verts, tris) -> Baked | None:
        verts = np.ascontiguousarray(verts, np.float32); tris = np.ascontiguousarray(tris, np.uint32)
        with tempfile.TemporaryDirectory() as d:
            scn = os.path.join(d, "g.scn")
            ok = self.L.ref_bake_arrays(_p(verts), verts.shape[0], _p(tris), tris.shape[0], scn.encode())
            if not ok:
                return None
            return Baked.read_bvh(os.path.join(d, "g.bvh"))

    def scene_geometry(self, scn_path):
        cnt = np.zeros(2, np.uint32)
        assert self.L.ref_scene_geometry(scn_path.encode(), None, None, _p(cnt))
        v = np.zeros((int(cnt[0]), 6), np.float32); t = np.zeros((int(cnt[1]), 3), np.uint32)
        assert self.L.ref_scene_geometry(scn_path.encode(), _p(v), _p(t), _p(cnt))
        return v, t

    def morton(self, verts, tris):
        verts = np.ascontiguousarray(verts, np.float32); tris = np.ascontiguousarray(tris, np.uint32)
        n = tris.shape[0]
        codes = np.zeros(n, np.uint64); perm = np.zeros(n, np.uint32); sb = np.zeros(6, np.float32)
        assert self.L.ref_morton(_p(verts), verts.shape[0], _p(tris), n, _p(codes), _p(perm), _p(sb))
        return codes, perm, sb

    def init_geos(self, verts, tris):
        v = np.ascontiguousarray(verts, np.float32).copy(); tris = np.ascontiguousarray(tris, np.uint32)
        assert self.L.ref_init_geos(_p(v), v.shape[0], _p(tris), tris.shape[0])
        return v

    def trace(self, baked: Baked, rays, threads: int = 1):
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "t.bvh")
            write_bvh(path, baked)
            assert self.L.ref_load(path.encode())
        out = np.zeros((n, 6), np.float32); tri = np.zeros(n, np.uint32); hit = np.zeros(n, np.uint8)
        self.L.ref_trace(_p(rays), n, _p(out), _p(tri), _p(hit), threads)
        return hit, out, tri

    def clip_triangle(self, v9, box6):
        v9 = np.ascontiguousarray(v9, np.float32); box6 = np.ascontiguousarray(box6, np.float32)
        out = np.zeros(6, np.float32)
        self.L.ref_clip_triangle(_p(v9), _p(box6), _p(out))
        return out

    def mesh_transform(self, translate, scale, q_wxyz, pos, nrm):
        """loadMesh's transform of imported positions and normals (bvh_IO.cpp:24-70, 221-224):
        (n, 6) float32 = x, y, z, nx, ny, nz."""
        pos = np.ascontiguousarray(pos, np.float32); nrm = np.ascontiguousarray(nrm, np.float32)
        out = np.zeros((pos.shape[0], 6), np.float32)
        self.L.ref_mesh_transform(_p(np.asarray(translate, np.float32)), float(scale),
                                  _p(np.asarray(q_wxyz, np.float32)), pos.shape[0], _p(pos), _p(nrm), _p(out))
        return out

    # ---- the path loop of src/main.cpp ----
    def scene_config(self, scn_path):
        """parseSceneConfig (main.cpp:218-285): (width, height), camera (13 floats: pos, fwd,
        right, up, tanHalfFovY), ambient, whether an ibl line named a map."""
        wh = np.zeros(2, np.int32); cam = np.zeros(13, np.float32); amb = np.zeros(3, np.float32)
        has_ibl = self.L.ref_scene_config(scn_path.encode(), _p(wh), _p(cam), _p(amb))
        return (int(wh[0]), int(wh[1])), cam, amb, bool(has_ibl)

    def camera_lookat(self, pos, target, fov_deg):
        cam = np.zeros(13, np.float32)
        self.L.ref_camera_lookat(_p(np.asarray(pos, np.float32)), _p(np.asarray(target, np.float32)),
                                 float(fov_deg), _p(cam))
        return cam

    def camera_quat(self, pos, q_wxyz, focal):
        cam = np.zeros(13, np.float32)
        self.L.ref_camera_quat(_p(np.asarray(pos, np.float32)), _p(np.asarray(q_wxyz, np.float32)), float(focal),
                               _p(cam))
        return cam

    def primary_rays(self, cam13, W, H, px, py, jx, jy):
        """primaryRay (main.cpp:69-83): (n, 8) rays = origin, tmin, dir, tmax."""
        px = np.ascontiguousarray(px, np.int32); py = np.ascontiguousarray(py, np.int32)
        jx = np.ascontiguousarray(jx, np.float32); jy = np.ascontiguousarray(jy, np.float32)
        out = np.zeros((px.shape[0], 8), np.float32)
        self.L.ref_primary_rays(_p(np.ascontiguousarray(cam13, np.float32)), int(W), int(H), px.shape[0], _p(px),
                                _p(py), _p(jx), _p(jy), _p(out))
        return out

    def cosine_dirs(self, u1, u2, normals):
        """toWorld(sampleCosineHemisphere(u1, u2), n) (main.cpp:123-141)."""
        u1 = np.ascontiguousarray(u1, np.float32); u2 = np.ascontiguousarray(u2, np.float32)
        nrm = np.ascontiguousarray(normals, np.float32)
        out = np.zeros((u1.shape[0], 3), np.float32)
        self.L.ref_cosine_dirs(u1.shape[0], _p(u1), _p(u2), _p(nrm), _p(out))
        return out

    def ibl_lookup(self, env_map, dirs):
        """IBL::sample (main.cpp:107-117) of an (h, w, 3) map."""
        em = np.ascontiguousarray(env_map, np.float32); d = np.ascontiguousarray(dirs, np.float32)
        out = np.zeros((d.shape[0], 3), np.float32)
        self.L.ref_ibl_lookup(_p(em), em.shape[1], em.shape[0], d.shape[0], _p(d), _p(out))
        return out

    def path_render(self, baked: Baked, cam13, W, H, spp, max_bounce=8, seed=1, env_map=None, rows=None,
                    threads: int = 1):
        """The reference's pixel loop and pathTrace (main.cpp:145-204, 339-365) over `baked`
        (loaded with the reference's loadBVH), one std::mt19937 per pixel. Returns the per-pixel
        mean and mean of squares, (rows, W, 3) float64, row 0 at the bottom."""
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "r.bvh")
            write_bvh(path, baked)
            assert self.L.ref_load(path.encode())
        r0, r1 = rows if rows is not None else (0, H)
        mean = np.zeros((r1 - r0, W, 3), np.float64); sq = np.zeros_like(mean)
        em = np.ascontiguousarray(env_map, np.float32) if env_map is not None else None
        eh, ew = (em.shape[0], em.shape[1]) if em is not None else (0, 0)
        ok = self.L.ref_path_render(_p(np.ascontiguousarray(cam13, np.float32)), int(W), int(H), int(spp),
                                    int(max_bounce), int(seed), _p(em), ew, eh, r0, r1 - r0, _p(mean), _p(sq),
                                    int(threads))
        assert ok
        return mean, sq


def write_bvh(path, baked: Baked):
    """Writes a .bvh v1 file with the layout of src/bvh/bvh_IO.cpp:256-265."""
    hdr = np.array([1, baked.nodes.shape[0], baked.tris.shape[0], baked.verts.shape[0]], "<u4")
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(np.ascontiguousarray(baked.nodes).tobytes())
        f.write(np.ascontiguousarray(baked.tris, "<u4").tobytes())
        f.write(np.ascontiguousarray(baked.verts, "<f4").tobytes())
