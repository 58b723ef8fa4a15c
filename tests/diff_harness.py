"""Test harness: rt_render / rt_adjoint wrapped as a torch.autograd.Function.

Parameters are indexed by INPUT triangle (what a user optimises); the library works on baked
triangles, so the forward gathers the albedo through the build's primitive ids and the
backward scatter-adds the baked gradients back (a triangle duplicated by a spatial split
receives the sum of its copies' gradients).
"""
import numpy as np
import torch

import rtb200


class RenderFunction(torch.autograd.Function):
    """image = render(albedo per input triangle (n, 3), emission per material (m, 3))."""

    @staticmethod
    def forward(ctx, albedo, emission, bvh, rcfg, scene_mats, mot_baked, prim):
        mats = _mats_with_emission(scene_mats, emission)
        talb = albedo.detach()[prim].contiguous()
        img, _ = bvh.render(rcfg, mats, mot_baked, tri_albedo=talb)
        ctx.save_for_backward(talb, mats)
        ctx.bvh, ctx.rcfg, ctx.mot, ctx.prim, ctx.n = bvh, rcfg, mot_baked, prim, albedo.shape[0]
        return img

    @staticmethod
    def backward(ctx, grad_img):
        talb, mats = ctx.saved_tensors
        g_baked, g_em = ctx.bvh.adjoint(ctx.rcfg, grad_img, mats, ctx.mot, tri_albedo=talb)
        g_alb = torch.zeros((ctx.n, 3), dtype=torch.float32, device=g_baked.device)
        g_alb.index_add_(0, ctx.prim, g_baked)
        return g_alb, g_em, None, None, None, None, None


def _mats_with_emission(scene_mats, emission):
    arr = torch.from_numpy(rtb200.materials_array(scene_mats)).cuda()
    arr[:, 3:6] = emission.detach()
    return arr.contiguous()


class DiffScene:
    """A built scene ready for RenderFunction."""

    def __init__(self, scene, preset: str = "lbvh30"):
        self.scene = scene
        self.bvh = rtb200.Bvh.build(scene.verts, scene.tris, preset)
        prim = self.bvh.prim_ids()
        self.prim = torch.from_numpy(prim.astype(np.int64)).cuda()
        self.mot = torch.from_numpy(scene.baked_materials(prim).astype(np.int32)).cuda()

    def emission(self):
        return torch.tensor([m.get("emission", (0.0, 0.0, 0.0)) for m in self.scene.mats], dtype=torch.float32,
                            device="cuda")

    def render(self, albedo, emission, rcfg):
        return RenderFunction.apply(albedo, emission, self.bvh, rcfg, self.scene.mats, self.mot, self.prim)
