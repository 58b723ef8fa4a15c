"""rtb200: host-side Python front end of librt_b200.so (BVH bake / load / trace and the path
loop of minsuk0519/ray-tracer on a B200). See api.py."""
from .api import (Bvh, BuildCfg, WavefrontParams, batch_arrays, Material, Mesh, RenderCfg, RtError, PRESETS, NODE_DTYPE, HIT_DTYPE, TRACE_ANY_HIT,
                  TRACE_CLOSEST, TRACE_WATERTIGHT, RENDER_PLAIN, RENDER_WAVEFRONT, bake_scene, header_symbols,
                  kernel_launches, last_error, lib, make_cfg, materials_array, read_hdr, render_cfg, scene_config,
                  write_hdr)

__all__ = ["Bvh", "BuildCfg", "WavefrontParams", "batch_arrays", "Material", "Mesh", "RenderCfg", "RtError", "PRESETS", "NODE_DTYPE", "HIT_DTYPE",
           "TRACE_ANY_HIT", "TRACE_CLOSEST", "TRACE_WATERTIGHT", "RENDER_PLAIN", "RENDER_WAVEFRONT", "bake_scene",
           "header_symbols", "kernel_launches", "last_error", "lib", "make_cfg", "materials_array", "read_hdr", "render_cfg",
           "scene_config", "write_hdr"]

from . import dist  # noqa: E402  (multi-process plumbing)
