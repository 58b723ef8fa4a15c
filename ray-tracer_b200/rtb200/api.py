"""Python host API over librt_b200.so (ctypes; the C ABI of include/rt_b200.h).

It mirrors the reference's bake / load / trace interface (src/bvh/bvh.hpp:45-52,
src/bvh/bvh_traverse.hpp:8-30) for numpy arrays (host memory) and torch CUDA tensors (device
memory). Every compute call runs the library's CUDA kernels; there is no CPU fallback: if
the library or a CUDA device is missing the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "librt_b200.so")
HEADER = os.path.join(os.path.dirname(PKG_DIR), "include", "rt_b200.h")

RT_HOST, RT_DEVICE = 0, 1
TRACE_CLOSEST, TRACE_ANY_HIT, TRACE_WATERTIGHT = 0, 1, 2
RENDER_PLAIN, RENDER_WAVEFRONT = 0, 1
HIT_FLAG_HIT, HIT_FLAG_OVERFLOW = 1, 2
STATUS = {0: "RT_OK", 1: "RT_E_INVALID", 2: "RT_E_IO", 3: "RT_E_FORMAT", 4: "RT_E_CAPACITY", 5: "RT_E_STACK",
          6: "RT_E_CUDA", 7: "RT_E_TIMEOUT", 8: "RT_E_EMPTY", 9: "RT_E_INDEX", 10: "RT_E_NOT_LOADED"}

NODE_DTYPE = np.dtype([("bmin", "<f4", 4), ("bmax", "<f4", 4), ("is_leaf", "u1"), ("pad0", "u1", 3),
                       ("a", "<u4"), ("b", "<u4"), ("pad1", "<u4")])
# one node of the 8-wide traversal layout (rt_bvh_wide_download)
WIDE_NODE_DTYPE = np.dtype([("p", "<f4", 3), ("meta", "<u4"), ("ref", "<u4", 8), ("cnt", "<u2", 8), ("qlo", "u1", (3, 8)),
                            ("qhi", "u1", (3, 8)), ("pad", "<u4", 4)])
HIT_DTYPE = np.dtype([("t", "<f4"), ("u", "<f4"), ("v", "<f4"), ("tri", "<u4"), ("n", "<f4", 3), ("flags", "<u4")])
assert NODE_DTYPE.itemsize == 48 and HIT_DTYPE.itemsize == 32


class RtError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class BuildCfg(C.Structure):
    _fields_ = [("lbvh_threshold", C.c_uint32), ("max_leaf", C.c_uint32), ("morton_bits", C.c_uint32),
                ("bins_min", C.c_uint32), ("bins_max", C.c_uint32), ("c_trav", C.c_float), ("c_isect", C.c_float),
                ("centroid_eps", C.c_float), ("spatial_eps", C.c_float), ("spatial_mult", C.c_float)]


class Material(C.Structure):
    _fields_ = [("albedo", C.c_float * 3), ("emission", C.c_float * 3), ("kind", C.c_uint32), ("pad", C.c_uint32)]


class Shading(C.Structure):
    _fields_ = [("mats", C.c_void_p), ("mat_of_tri", C.c_void_p), ("tri_albedo", C.c_void_p), ("env_map", C.c_void_p),
                ("n_mats", C.c_uint32), ("env_w", C.c_uint32), ("env_h", C.c_uint32), ("pad", C.c_uint32)]


class WavefrontParams(C.Structure):
    _fields_ = [("trace_block", C.c_uint32), ("chunk_paths", C.c_uint32), ("stack_depth", C.c_uint32),
                ("shade_block", C.c_uint32)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class RenderCfg(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("max_bounce", C.c_uint32),
                ("rr_after", C.c_int32), ("env_kind", C.c_uint32), ("env_color", C.c_float * 3),
                ("cam_pos", C.c_float * 3), ("cam_fwd", C.c_float * 3), ("cam_right", C.c_float * 3),
                ("cam_up", C.c_float * 3), ("tan_half_fov_y", C.c_float), ("seed", C.c_uint32),
                ("sample_offset", C.c_uint32)]


# Build presets: the reference's defaults and the parameter sets of the benchmark builds.
PRESETS = {
    "hybrid":   dict(lbvh_threshold=64, max_leaf=16, morton_bits=21),        # the reference as shipped
    "lbvh63":   dict(lbvh_threshold=0, max_leaf=16, morton_bits=21),         # pure Morton split, 63-bit codes
    "lbvh30":   dict(lbvh_threshold=0, max_leaf=16, morton_bits=10),         # pure Morton split, 30-bit codes
    "lbvh63l4": dict(lbvh_threshold=0, max_leaf=4, morton_bits=21),
    "sah4":     dict(lbvh_threshold=0xFFFFFFFF, max_leaf=4, morton_bits=21), # binned SAH + spatial splits, leaf 4
    "sah16":    dict(lbvh_threshold=0xFFFFFFFF, max_leaf=16, morton_bits=21),
    "sah4ns":   dict(lbvh_threshold=0xFFFFFFFF, max_leaf=4, morton_bits=21, spatial_eps=3.0e38),  # no spatial splits
}

_lib = None


def lib():
    """Loads librt_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `make -C ray-tracer_b200`")
        L = C.CDLL(LIB_PATH)
        vp, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
        L.rt_build_cfg_default.argtypes = [vp]
        L.rt_build.argtypes = [vp, u32, vp, u32, i32, vp, vp, vp]
        L.rt_rebuild.argtypes = [vp, vp, u32, vp, u32, i32, vp, vp]
        L.rt_load_bvh.argtypes = [C.c_char_p, vp]
        L.rt_write_bvh.argtypes = [vp, C.c_char_p]
        L.rt_bvh_from_arrays.argtypes = [vp, u32, vp, u32, vp, u32, vp]
        L.rt_bvh_counts.argtypes = [vp, vp]
        L.rt_bvh_download.argtypes = [vp, vp, vp, vp]
        L.rt_bvh_download_async.argtypes = [vp, vp, vp, vp, vp]
        L.rt_bvh_wide_download.argtypes = [vp, vp, vp]
        L.rt_bvh_prim_ids.argtypes = [vp, vp, i32]
        L.rt_bvh_stats.argtypes = [vp, vp]
        L.rt_bvh_free.argtypes = [vp]
        L.rt_bvh_profile.argtypes = [vp, i32]
        L.rt_bvh_stage_ms.argtypes = [vp, vp]
        L.rt_trace.argtypes = [vp, vp, vp, u64, u32, vp]
        L.rt_bvh_trace_loop.argtypes = [vp, i32]
        L.rt_trace_host.argtypes = [vp, vp, vp, u64, u32]
        L.rt_render.argtypes = [vp, vp, vp, u32, vp, i32, vp, vp, vp]
        L.rt_render_ex.argtypes = [vp, vp, vp, i32, vp, vp, vp]
        L.rt_adjoint.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        L.rt_build_batch.argtypes = [vp, vp, vp, vp, u32, i32, vp, vp, vp]
        L.rt_rebuild_batch.argtypes = [vp, vp, vp, vp, vp, u32, i32, vp, vp]
        L.rt_write_hdr.argtypes = [C.c_char_p, vp, u32, u32, i32]
        L.rt_read_hdr.argtypes = [C.c_char_p, vp, vp, vp]
        L.rt_scene_config.argtypes = [C.c_char_p, vp, C.c_char_p, u32]
        L.rt_render_host.argtypes = [vp, vp, vp, i32, vp]
        L.rt_bvh_scenes.argtypes = [vp, vp, vp]
        L.rt_bvh_depth.argtypes = [vp, vp]
        L.rt_render_batch.argtypes = [vp, vp, u32, vp, vp, vp, vp, vp]
        L.rt_autotune_wavefront.argtypes = [vp, vp, u32, vp, vp, vp]
        L.rt_camera_lookat.argtypes = [vp, vp, C.c_float, vp]
        L.rt_camera_quat.argtypes = [vp, vp, C.c_float, vp]
        L.rt_mesh_create.restype = vp
        L.rt_mesh_free.argtypes = [vp]
        L.rt_mesh_add_sphere.argtypes = [vp, C.c_float, C.c_float, C.c_float, C.c_float, i32, i32]
        L.rt_mesh_add_box.argtypes = [vp] + [C.c_float] * 10
        L.rt_mesh_read_scene.argtypes = [vp, C.c_char_p]
        L.rt_mesh_counts.argtypes = [vp, vp]
        L.rt_mesh_vertices.restype = vp
        L.rt_mesh_vertices.argtypes = [vp]
        L.rt_mesh_triangles.restype = vp
        L.rt_mesh_triangles.argtypes = [vp]
        L.rt_bake_scene.argtypes = [C.c_char_p, C.c_char_p, vp]
        L.rt_last_error.restype = C.c_char_p
        L.rt_version.restype = C.c_char_p
        L.rt_kernel_launches.restype = u64
        L.rt_device_allocations.restype = u64
        L.rt_device_sync.argtypes = [vp]
        L.rt_morton_order_noalloc.argtypes = [vp, u32, vp, u32, u32, vp, vp]
        _lib = L
    return _lib


def header_symbols(path: str = HEADER) -> list[str]:
    """Names of the functions include/rt_b200.h declares."""
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(rt_[a-z0-9_]+)\s*\(", txt)))


def _check(code: int):
    if code != 0:
        raise RtError(code, lib().rt_last_error().decode(errors="replace"))


def last_error() -> str:
    return lib().rt_last_error().decode(errors="replace")


def kernel_launches() -> int:
    return int(lib().rt_kernel_launches())


def device_allocations() -> int:
    """Device allocations (cudaMalloc) the library has made so far in this process."""
    return int(lib().rt_device_allocations())


def make_cfg(preset: str = "hybrid", **kw) -> BuildCfg:
    c = BuildCfg()
    lib().rt_build_cfg_default(C.byref(c))
    for k, v in {**PRESETS[preset], **kw}.items():
        setattr(c, k, v)
    return c


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x):
    if x is None:
        return None
    if _is_torch(x):
        return C.c_void_p(x.data_ptr())
    return x.ctypes.data_as(C.c_void_p)


def _stream_ptr(stream, torch_tensors: bool = False):
    """The stream handle for a call. None with torch tensors: torch's current stream, so the
    work is ordered with the torch operations around it; None otherwise: the library's own
    stream. torch reports its legacy default stream as 0, which the C ABI reads as "the
    library's stream", so it is passed as cudaStreamLegacy (1) instead."""
    if stream is None:
        if not torch_tensors:
            return None
        import torch
        stream = torch.cuda.current_stream()
    h = int(stream.cuda_stream) if hasattr(stream, "cuda_stream") else int(stream)
    return C.c_void_p(h if h != 0 else 1)


class Bvh:
    """A device-resident BVH (an rt_bvh handle)."""

    def __init__(self, handle):
        self.h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle

    # -- construction ------------------------------------------------------------------
    @staticmethod
    def build(verts, tris, cfg: BuildCfg | str | None = None, stream=None) -> "Bvh":
        """verts: (V, 6) float32 (x y z nx ny nz), tris: (N, 3) uint32; numpy (host) or torch
        CUDA tensors (device)."""
        if isinstance(cfg, str):
            cfg = make_cfg(cfg)
        verts, tris, where = _geometry(verts, tris)
        out = C.c_void_p()
        _check(lib().rt_build(_ptr(verts), int(verts.shape[0]), _ptr(tris), int(tris.shape[0]), where,
                              C.byref(cfg) if cfg is not None else None, _stream_ptr(stream, where == RT_DEVICE),
                              C.byref(out)))
        return Bvh(out)

    def rebuild(self, verts, tris, cfg: BuildCfg | str | None = None, stream=None):
        if isinstance(cfg, str):
            cfg = make_cfg(cfg)
        verts, tris, where = _geometry(verts, tris)
        _check(lib().rt_rebuild(self.h, _ptr(verts), int(verts.shape[0]), _ptr(tris), int(tris.shape[0]), where,
                                C.byref(cfg) if cfg is not None else None, _stream_ptr(stream, where == RT_DEVICE)))

    @staticmethod
    def build_batch(verts, tris, vert_offsets, tri_offsets, cfg: BuildCfg | str | None = None, stream=None) -> "Bvh":
        """Many scenes in one build (rt_build_batch): verts / tris concatenated over the scenes
        with vertex indices local to each scene, offsets (n_scenes + 1,) ascending from 0.
        batch_arrays() makes these from a list of (verts, tris)."""
        if isinstance(cfg, str):
            cfg = make_cfg(cfg)
        verts, tris, where = _geometry(verts, tris)
        vo = np.ascontiguousarray(vert_offsets, np.uint32)
        to = np.ascontiguousarray(tri_offsets, np.uint32)
        out = C.c_void_p()
        _check(lib().rt_build_batch(_ptr(verts), _ptr(vo), _ptr(tris), _ptr(to), int(to.shape[0] - 1), where,
                                    C.byref(cfg) if cfg is not None else None, _stream_ptr(stream, where == RT_DEVICE),
                                    C.byref(out)))
        return Bvh(out)

    def rebuild_batch(self, verts, tris, vert_offsets, tri_offsets, cfg: BuildCfg | str | None = None, stream=None):
        if isinstance(cfg, str):
            cfg = make_cfg(cfg)
        verts, tris, where = _geometry(verts, tris)
        vo = np.ascontiguousarray(vert_offsets, np.uint32)
        to = np.ascontiguousarray(tri_offsets, np.uint32)
        _check(lib().rt_rebuild_batch(self.h, _ptr(verts), _ptr(vo), _ptr(tris), _ptr(to), int(to.shape[0] - 1), where,
                                      C.byref(cfg) if cfg is not None else None, _stream_ptr(stream, where == RT_DEVICE)))

    def scenes(self):
        """(n_scenes, 4) uint32: root node, node count, first triangle, triangle count per scene."""
        n = C.c_uint32(0)
        _check(lib().rt_bvh_scenes(self.h, C.byref(n), None))
        info = np.zeros((n.value, 4), np.uint32)
        if n.value:
            _check(lib().rt_bvh_scenes(self.h, C.byref(n), _ptr(info)))
        return info

    def scene_arrays(self, s: int, vert_offsets, download=None):
        """Scene s of a batched build in its own numbering: (nodes, tris, verts) as rt_build of
        that scene alone lays them out."""
        nodes, tris, verts = download if download is not None else self.download()
        root, nn, t0, nt = (int(x) for x in self.scenes()[s])
        v0, v1 = int(vert_offsets[s]), int(vert_offsets[s + 1])
        sn = nodes[root:root + nn].copy()
        inner = sn["is_leaf"] == 0
        sn["a"] = np.where(inner, sn["a"] - root, sn["a"] - t0)
        sn["b"] = np.where(inner, sn["b"] - root, sn["b"])
        return sn, tris[t0:t0 + nt] - np.uint32(v0), verts[v0:v1]

    def depth(self) -> int:
        d = C.c_uint32(0)
        _check(lib().rt_bvh_depth(self.h, C.byref(d)))
        return int(d.value)

    @staticmethod
    def load(path: str) -> "Bvh":
        out = C.c_void_p()
        _check(lib().rt_load_bvh(path.encode(), C.byref(out)))
        return Bvh(out)

    @staticmethod
    def from_arrays(nodes, tris, verts) -> "Bvh":
        nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
        tris = np.ascontiguousarray(tris, np.uint32)
        verts = np.ascontiguousarray(verts, np.float32)
        out = C.c_void_p()
        _check(lib().rt_bvh_from_arrays(_ptr(nodes), nodes.shape[0], _ptr(tris), tris.shape[0], _ptr(verts),
                                        verts.shape[0], C.byref(out)))
        return Bvh(out)

    def free(self):
        if self.h:
            lib().rt_bvh_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    # -- inspection --------------------------------------------------------------------
    def counts(self):
        c = np.zeros(3, np.uint32)
        _check(lib().rt_bvh_counts(self.h, _ptr(c)))
        return int(c[0]), int(c[1]), int(c[2])

    def download(self):
        """(nodes, tris, verts) in the .bvh v1 layout."""
        nn, nt, nv = self.counts()
        nodes = np.zeros(nn, NODE_DTYPE)
        tris = np.zeros((nt, 3), np.uint32)
        verts = np.zeros((nv, 6), np.float32)
        _check(lib().rt_bvh_download(self.h, _ptr(nodes), _ptr(tris), _ptr(verts)))
        return nodes, tris, verts

    def prim_ids(self):
        _, nt, _ = self.counts()
        out = np.zeros(nt, np.uint32)
        _check(lib().rt_bvh_prim_ids(self.h, _ptr(out), RT_HOST))
        return out

    def stats(self):
        s = np.zeros(8, np.uint32)
        _check(lib().rt_bvh_stats(self.h, _ptr(s)))
        return dict(spatial_taken=int(s[0]), spatial_refused=int(s[1]), sah_roots=int(s[2]), inner=int(s[3]),
                    leaves=int(s[4]))

    def profile(self, enable: bool = True):
        """Stage timing (CUDA events on the build stream) for later rebuilds of this handle."""
        _check(lib().rt_bvh_profile(self.h, 1 if enable else 0))

    def stage_ms(self):
        ms = np.zeros(8, np.float32)
        _check(lib().rt_bvh_stage_ms(self.h, _ptr(ms)))
        names = ["prep", "sort", "topology", "sah", "emit", "layout", "total"]
        return {k: float(ms[i]) for i, k in enumerate(names)}

    def write(self, path: str):
        _check(lib().rt_write_bvh(self.h, path.encode()))

    def trace_loop(self, form: int = -1):
        """Traversal form: 0 one-loop, 1 while-while, -1 the default choice by leaf size (all three
        the reference's visiting order); 2 the 8-wide layout (same closest distance, ties may
        report another triangle; kept up to date across rebuilds)."""
        _check(lib().rt_bvh_trace_loop(self.h, int(form)))

    def wide_nodes(self):
        """The 8-wide layout (after trace_loop(2)) as a WIDE_NODE_DTYPE array."""
        n = C.c_uint32(0)
        _check(lib().rt_bvh_wide_download(self.h, None, C.byref(n)))
        out = np.zeros(n.value, WIDE_NODE_DTYPE)
        _check(lib().rt_bvh_wide_download(self.h, _ptr(out), C.byref(n)))
        return out

    # -- tracing -----------------------------------------------------------------------
    def trace(self, rays, flags: int = TRACE_CLOSEST, stream=None):
        """rays: (n, 8) float32 (o.xyz, tmin, d.xyz, tmax). numpy in -> structured HIT_DTYPE
        numpy out (host copies inside); torch CUDA in -> (n, 8) float32 tensor of rt_hit
        records out (device)."""
        if _is_torch(rays):
            import torch
            assert rays.is_cuda and rays.dtype == torch.float32 and rays.shape[-1] == 8
            rays = rays.contiguous()
            hits = torch.empty_like(rays)
            code = lib().rt_trace(self.h, _ptr(rays), _ptr(hits), int(rays.shape[0]), flags, _stream_ptr(stream, True))
            if code not in (0, 5):
                _check(code)
            return hits
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros(rays.shape[0], HIT_DTYPE)
        code = lib().rt_trace_host(self.h, _ptr(rays), _ptr(hits), int(rays.shape[0]), flags)
        if code not in (0, 5):
            _check(code)
        return hits

    def render(self, rcfg: RenderCfg, mats=None, mat_of_tri=None, mode: int = RENDER_PLAIN, want_sq: bool = False,
               stream=None, tri_albedo=None, env_map=None):
        """Returns (rgb, rgb2) torch CUDA tensors (H, W, 3); mats: list of dicts or None;
        mat_of_tri: material index per baked triangle (numpy / torch); tri_albedo: (n_tris, 3)
        float32 albedo per baked triangle (numpy / torch), replacing the materials' albedo; env_map:
        (h, w, 3) float32 equirectangular environment for env_kind 2."""
        import torch
        rgb = torch.empty((rcfg.height, rcfg.width, 3), dtype=torch.float32, device="cuda")
        rgb2 = torch.empty_like(rgb) if want_sq else None
        sh, keep = _shading(mats, mat_of_tri, tri_albedo, env_map)
        _check(lib().rt_render_ex(self.h, C.byref(rcfg), C.byref(sh), mode, _ptr(rgb), _ptr(rgb2),
                                  _stream_ptr(stream, True)))
        del keep
        return rgb, rgb2

    def adjoint(self, rcfg: RenderCfg, d_rgb, mats=None, mat_of_tri=None, tri_albedo=None, stream=None):
        """Path-replay adjoint of render(): d_rgb = dLoss/d(rgb) as an (H, W, 3) float32 CUDA
        tensor. Returns (grad_albedo (n_tris, 3), grad_emission (n_mats, 3) or None) as float32
        CUDA tensors, indexed like tri_albedo / mats."""
        import torch
        _, nt, _ = self.counts()
        d_rgb = d_rgb.contiguous().to(torch.float32)
        assert d_rgb.is_cuda and d_rgb.numel() == rcfg.width * rcfg.height * 3
        g_alb = torch.zeros((nt, 3), dtype=torch.float32, device="cuda")
        g_em = torch.zeros((len(mats), 3), dtype=torch.float32, device="cuda") if mats is not None else None
        sh, keep = _shading(mats, mat_of_tri, tri_albedo)
        _check(lib().rt_adjoint(self.h, C.byref(rcfg), C.byref(sh), _ptr(d_rgb), _ptr(g_alb), _ptr(g_em),
                                _stream_ptr(stream, True)))
        del keep
        return g_alb, g_em


    def render_batch(self, rcfgs, mats=None, mat_of_tri=None, params: WavefrontParams | None = None, want_sq=False,
                     stream=None, tri_albedo=None):
        """All scenes of a batched handle in one wavefront render: rcfgs = one RenderCfg per scene
        (camera and seed; the rest from rcfgs[0]). Returns (rgb, rgb2) (n_scenes, H, W, 3)."""
        import torch
        n = len(rcfgs)
        arr = (RenderCfg * n)(*rcfgs)
        c0 = rcfgs[0]
        rgb = torch.empty((n, c0.height, c0.width, 3), dtype=torch.float32, device="cuda")
        rgb2 = torch.empty_like(rgb) if want_sq else None
        sh, keep = _shading(mats, mat_of_tri, tri_albedo)
        _check(lib().rt_render_batch(self.h, arr, n, C.byref(sh), C.byref(params) if params is not None else None,
                                     _ptr(rgb), _ptr(rgb2), _stream_ptr(stream, True)))
        del keep
        return rgb, rgb2

    def autotune(self, rcfgs, mats=None, mat_of_tri=None, stream=None) -> WavefrontParams:
        n = len(rcfgs)
        arr = (RenderCfg * n)(*rcfgs)
        best = WavefrontParams()
        sh, keep = _shading(mats, mat_of_tri, None)
        _check(lib().rt_autotune_wavefront(self.h, arr, n, C.byref(sh), C.byref(best), _stream_ptr(stream, True)))
        del keep
        return best


def write_hdr(path: str, rgb, flip_y: bool = False):
    """Writes an (h, w, 3) float32 image as a Radiance RGBE .hdr file."""
    a = np.ascontiguousarray(rgb, np.float32)
    _check(lib().rt_write_hdr(path.encode(), _ptr(a), int(a.shape[1]), int(a.shape[0]), 1 if flip_y else 0))


def read_hdr(path: str) -> np.ndarray:
    """Reads a Radiance RGBE .hdr file into an (h, w, 3) float32 array (file row order)."""
    w, h = C.c_uint32(0), C.c_uint32(0)
    _check(lib().rt_read_hdr(path.encode(), None, C.byref(w), C.byref(h)))
    out = np.zeros((h.value, w.value, 3), np.float32)
    _check(lib().rt_read_hdr(path.encode(), _ptr(out), C.byref(w), C.byref(h)))
    return out


def scene_config(path: str, rcfg: RenderCfg | None = None):
    """(RenderCfg with the .scn file's screen size and camera, ibl path or '')."""
    c = rcfg if rcfg is not None else render_cfg(1, 1, 1)
    buf = C.create_string_buffer(4096)
    _check(lib().rt_scene_config(path.encode(), C.byref(c), buf, 4096))
    return c, buf.value.decode()


def batch_arrays(parts):
    """(verts, tris, vert_offsets, tri_offsets) for rt_build_batch from a list of (verts, tris)
    with per-scene vertex indices."""
    vo = np.zeros(len(parts) + 1, np.uint32)
    to = np.zeros(len(parts) + 1, np.uint32)
    for i, (v, t) in enumerate(parts):
        vo[i + 1] = vo[i] + v.shape[0]
        to[i + 1] = to[i] + t.shape[0]
    verts = np.concatenate([np.asarray(v, np.float32) for v, _ in parts])
    tris = np.concatenate([np.asarray(t, np.uint32) for _, t in parts])
    return verts, tris, vo, to


def materials_array(mats) -> np.ndarray:
    """rt_material records (n, 8) float32 from a list of dicts (albedo, emission, kind)."""
    arr = np.zeros((len(mats), 8), np.float32)
    for i, m in enumerate(mats):
        arr[i, 0:3] = m["albedo"]
        arr[i, 3:6] = m.get("emission", (0.0, 0.0, 0.0))
        arr[i, 6:8].view(np.uint32)[0] = int(m.get("kind", 0))
    return arr


def _device_u32(x):
    import torch
    if x is None:
        return None
    if _is_torch(x):
        return x.contiguous().cuda()
    return torch.from_numpy(np.ascontiguousarray(x, np.uint32).view(np.int32)).cuda()


def _shading(mats, mat_of_tri, tri_albedo, env_map=None):
    """An rt_shading record over device copies of the inputs (kept alive by the caller)."""
    import torch
    sh = Shading()
    keep = []
    if env_map is not None:
        em = env_map if _is_torch(env_map) else torch.from_numpy(np.ascontiguousarray(env_map, np.float32))
        em = em.to(device="cuda", dtype=torch.float32).contiguous()
        keep.append(em)
        sh.env_map, sh.env_h, sh.env_w = em.data_ptr(), int(em.shape[0]), int(em.shape[1])
    if mats is not None:
        dm = mats.contiguous().cuda() if _is_torch(mats) else torch.from_numpy(materials_array(mats)).cuda()
        keep.append(dm)
        sh.mats, sh.n_mats = dm.data_ptr(), int(dm.shape[0])
        if mat_of_tri is not None:
            dmot = _device_u32(mat_of_tri)
            keep.append(dmot)
            sh.mat_of_tri = dmot.data_ptr()
    if tri_albedo is not None:
        ta = tri_albedo.detach() if _is_torch(tri_albedo) else torch.from_numpy(np.ascontiguousarray(tri_albedo, np.float32))
        ta = ta.to(device="cuda", dtype=torch.float32).contiguous()
        keep.append(ta)
        sh.tri_albedo = ta.data_ptr()
    return sh, keep


def _geometry(verts, tris):
    if _is_torch(verts):
        import torch
        assert verts.is_cuda and tris.is_cuda
        verts = verts.contiguous().to(torch.float32)
        tris = tris.contiguous()
        assert tris.element_size() == 4
        return verts, tris, RT_DEVICE
    return np.ascontiguousarray(verts, np.float32), np.ascontiguousarray(tris, np.uint32), RT_HOST


def render_cfg(width, height, spp, max_bounce=8, rr_after=2, env_kind=0, env_color=(0.0, 0.0, 0.0), seed=1,
               sample_offset=0, lookat=None, quat=None) -> RenderCfg:
    """Render settings; lookat=(pos, target, fov_deg) or quat=(pos, (w, x, y, z), focal)
    (src/main.cpp:43-66). Defaults are the reference's: 8 bounces, roulette after bounce 2,
    sky background."""
    c = RenderCfg()
    c.width, c.height, c.spp, c.max_bounce, c.rr_after, c.env_kind = width, height, spp, max_bounce, rr_after, env_kind
    c.env_color[:] = list(env_color)
    c.seed, c.sample_offset = seed, sample_offset
    if quat is not None:
        pos, q, focal = quat
        lib().rt_camera_quat(_ptr(np.asarray(pos, np.float32)), _ptr(np.asarray(q, np.float32)), float(focal), C.byref(c))
    else:
        pos, target, fov = lookat if lookat is not None else ((0.0, 1.0, -5.0), (0.0, 0.0, 0.0), 60.0)
        lib().rt_camera_lookat(_ptr(np.asarray(pos, np.float32)), _ptr(np.asarray(target, np.float32)), float(fov),
                               C.byref(c))
    return c


class Mesh:
    """Host geometry built with the reference's generators (rt_mesh_*)."""

    def __init__(self):
        self.h = C.c_void_p(lib().rt_mesh_create())

    def __del__(self):
        try:
            if self.h:
                lib().rt_mesh_free(self.h)
        except Exception:
            pass

    def add_sphere(self, center, radius, rings=16, sectors=32):
        _check(lib().rt_mesh_add_sphere(self.h, *[float(x) for x in center], float(radius), int(rings), int(sectors)))
        return self

    def add_box(self, center, half, q_xyzw=(0.0, 0.0, 0.0, 1.0)):
        _check(lib().rt_mesh_add_box(self.h, *[float(x) for x in center], *[float(x) for x in half],
                                     *[float(x) for x in q_xyzw]))
        return self

    def read_scene(self, path: str):
        _check(lib().rt_mesh_read_scene(self.h, path.encode()))
        return self

    def arrays(self):
        c = np.zeros(2, np.uint32)
        _check(lib().rt_mesh_counts(self.h, _ptr(c)))
        nv, nt = int(c[0]), int(c[1])
        v = np.zeros((nv, 6), np.float32)
        t = np.zeros((nt, 3), np.uint32)
        if nv:
            C.memmove(v.ctypes.data, lib().rt_mesh_vertices(self.h), nv * 24)
        if nt:
            C.memmove(t.ctypes.data, lib().rt_mesh_triangles(self.h), nt * 12)
        return v, t


NOALLOC_MAX_TRIS = 65536


def morton_order_noalloc(dverts, dtris, perm_out, morton_bits: int = 21, stream=None):
    """rt_morton_order_noalloc on torch CUDA tensors: writes the Morton-sorted original triangle
    indices into perm_out (int32/uint32, n_tris entries) without any device allocation, for
    callers that may not allocate while they run (see include/rt_b200.h). The tensors must be
    contiguous: making a copy would allocate, so non-contiguous input is refused."""
    for name, x in (("verts", dverts), ("tris", dtris), ("perm_out", perm_out)):
        if not x.is_cuda or not x.is_contiguous():
            raise ValueError(f"{name} must be a contiguous CUDA tensor")
    if dtris.element_size() != 4 or perm_out.element_size() != 4 or perm_out.numel() < dtris.shape[0]:
        raise ValueError("tris and perm_out must hold 32-bit integers, perm_out at least n_tris of them")
    _check(lib().rt_morton_order_noalloc(_ptr(dverts), int(dverts.shape[0]), _ptr(dtris), int(dtris.shape[0]),
                                         int(morton_bits), _ptr(perm_out), _stream_ptr(stream, True)))
    return perm_out


def bake_scene(scn_path: str, out_bvh: str | None = None, cfg: BuildCfg | str | None = None):
    """bvh::bakeBVH: .scn -> GPU build -> .bvh."""
    if isinstance(cfg, str):
        cfg = make_cfg(cfg)
    _check(lib().rt_bake_scene(scn_path.encode(), out_bvh.encode() if out_bvh else None,
                               C.byref(cfg) if cfg is not None else None))
