"""GPU adjoint (rt_adjoint, path-replay backpropagation) against
  * the oracle's FP64 adjoint (stored paths, explicit products) on a small case;
  * central finite differences of rt_render (h = 1e-3, the same counter-based random numbers
    in both perturbed renders) of an L2 image loss, on 64 random albedo parameters and the
    light's radiance;
and the torch.autograd.Function harness (tests/diff_harness.py) end to end.
Per-triangle albedo in the forward render is checked against the oracle too."""
import numpy as np
import pytest
import torch

import rtb200
from diff_harness import DiffScene
from oracle import Baked
from rtb200 import scenes
from test_gpu_render import compare, orc_cfg_from

pytestmark = pytest.mark.gpu


def small_scene(level=2):
    cv, ct, cid = scenes.cornell()
    iv, it = scenes.icosphere(level, center=(0.0, -0.4, 0.2), radius=0.45, seed=21)
    v, t, _ = scenes.concat([(cv, ct), (iv, it)])
    obj = np.concatenate([cid, np.full(it.shape[0], 6, np.uint32)])
    mats = [dict(albedo=(0.75, 0.75, 0.75)), dict(albedo=(0.75, 0.75, 0.75)), dict(albedo=(0.75, 0.75, 0.75)),
            dict(albedo=(0.65, 0.1, 0.1)), dict(albedo=(0.1, 0.6, 0.15)),
            dict(albedo=(0.0, 0.0, 0.0), emission=(15.0, 15.0, 15.0)), dict(albedo=(0.5, 0.5, 0.5))]
    return scenes.Scene(v, t, obj, mats, np.arange(7), scenes.CORNELL_LOOKAT)


def rcfg(w, h, spp, max_bounce=3, rr_after=-1, seed=9):
    return rtb200.render_cfg(w, h, spp, max_bounce=max_bounce, rr_after=rr_after, env_kind=1, seed=seed,
                             lookat=scenes.CORNELL_LOOKAT)


@pytest.mark.parametrize("rr_after", [-1, 1])
def test_adjoint_matches_oracle_fp64(orc, rr_after):
    sc = small_scene()
    b = rtb200.Bvh.build(sc.verts, sc.tris, "lbvh30")
    prim = b.prim_ids()
    mot = sc.baked_materials(prim)
    rng = np.random.default_rng(3)
    talb = rng.uniform(0.2, 0.8, size=(sc.tris.shape[0], 3)).astype(np.float32)[prim]
    rc = rcfg(40, 32, 8, max_bounce=4, rr_after=rr_after)
    d = rng.uniform(0.5, 1.5, size=(rc.height, rc.width, 3)).astype(np.float32)
    g, e = b.adjoint(rc, torch.from_numpy(d).cuda(), sc.mats, mot, tri_albedo=talb)
    nodes, tris, verts = b.download()
    go, eo = orc.adjoint(Baked(nodes, tris, verts), orc_cfg_from(rc), d, sc.mats, mot, talb, threads=8)
    g, e = g.cpu().numpy().astype(np.float64), e.cpu().numpy().astype(np.float64)
    # the same paths on both sides except where device and host cosf/sinf differ by an ulp
    rel = np.linalg.norm(g - go) / np.linalg.norm(go)
    assert rel < 2e-3, rel
    close = np.abs(g - go) <= 1e-4 * np.abs(go) + 1e-6 * np.abs(go).max()
    assert close.mean() > 0.97, close.mean()
    assert np.allclose(e, eo, rtol=2e-3, atol=1e-6 * np.abs(eo).max()), (e, eo)


def test_forward_tri_albedo_matches_oracle(orc):
    sc = small_scene()
    b = rtb200.Bvh.build(sc.verts, sc.tris, "lbvh63")
    prim = b.prim_ids()
    mot = sc.baked_materials(prim)
    talb = np.random.default_rng(4).uniform(0.2, 0.8, size=(sc.tris.shape[0], 3)).astype(np.float32)[prim]
    rc = rcfg(40, 32, 16, max_bounce=4, rr_after=2)
    rgb, rgb2 = b.render(rc, sc.mats, mot, want_sq=True, tri_albedo=talb)
    nodes, tris, verts = b.download()
    ref, ref2 = orc.render(Baked(nodes, tris, verts), orc_cfg_from(rc), sc.mats, mot, threads=8, want_sq=True,
                           tri_albedo=talb)
    compare(rgb, rgb2, ref, ref2, rc.spp, "tri albedo")
    w, _ = b.render(rc, sc.mats, mot, mode=rtb200.RENDER_WAVEFRONT, tri_albedo=talb)
    assert np.allclose(w.cpu().numpy(), rgb.cpu().numpy(), rtol=1e-5, atol=1e-6)


def fd_case(n_ico_tris=5120, w=96, h=96, spp=8):
    sc, init, gt = scenes.diff_scene(n_ico_tris=n_ico_tris)
    ds = DiffScene(sc)
    rc = rcfg(w, h, spp, max_bounce=4)
    em = ds.emission()
    with torch.no_grad():
        target = ds.render(torch.from_numpy(gt).cuda(), em, rcfg(w, h, 4 * spp, max_bounce=4, seed=77))
    return ds, rc, torch.from_numpy(init).cuda(), em, target


def l2(img, target):
    return ((img.double() - target.double()) ** 2).sum()


def test_adjoint_matches_central_differences():
    ds, rc, alb, em, target = fd_case()
    a = alb.clone().requires_grad_(True)
    e = em.clone().requires_grad_(True)
    l2(ds.render(a, e, rc), target).backward()
    g_alb, g_em = a.grad.cpu().numpy(), e.grad.cpu().numpy()
    # 64 random albedo parameters among the triangles the camera sees (a zero gradient is
    # trivially matched), and the light's radiance
    seen = np.flatnonzero(np.abs(g_alb).max(axis=1) > 1e-3 * np.abs(g_alb).max())
    rng = np.random.default_rng(12)
    picks = [(int(t), int(c)) for t, c in zip(rng.choice(seen, 64, replace=False), rng.integers(0, 3, 64))]
    hstep = 1e-3
    errs = []
    with torch.no_grad():
        for t, c in picks:
            ap, am = alb.clone(), alb.clone()
            ap[t, c] += hstep; am[t, c] -= hstep
            fd = (l2(ds.render(ap, em, rc), target) - l2(ds.render(am, em, rc), target)).item() / (2 * hstep)
            errs.append(abs(fd - g_alb[t, c]) / max(abs(fd), 1e-12))
        light = 5
        for c in range(3):
            ep, emn = em.clone(), em.clone()
            ep[light, c] += hstep; emn[light, c] -= hstep
            fd = (l2(ds.render(alb, ep, rc), target) - l2(ds.render(alb, emn, rc), target)).item() / (2 * hstep)
            errs.append(abs(fd - g_em[light, c]) / max(abs(fd), 1e-12))
    errs = np.array(errs)
    assert np.median(errs) < 1e-3, np.median(errs)
    assert (errs <= 1e-2).mean() >= 0.95, np.sort(errs)[-8:]


def test_autograd_harness_descends():
    """A few gradient steps on the albedo through RenderFunction reduce the L2 loss."""
    ds, rc, alb, em, target = fd_case(n_ico_tris=1280, w=64, h=64, spp=16)
    a = alb.clone().requires_grad_(True)
    opt = torch.optim.SGD([a], lr=0.0)
    losses = []
    for it in range(6):
        opt.zero_grad()
        loss = l2(ds.render(a, em, rc), target)
        loss.backward()
        if it == 0:
            opt.param_groups[0]["lr"] = 0.05 / float(a.grad.abs().max())
        opt.step()
        with torch.no_grad():
            a.clamp_(0.0, 1.0)
        losses.append(loss.item())
    assert losses[-1] < 0.9 * losses[0], losses


def test_adjoint_skips_zero_weight_pixels_and_validates():
    sc = small_scene(1)
    b = rtb200.Bvh.build(sc.verts, sc.tris, "lbvh30")
    mot = sc.baked_materials(b.prim_ids())
    rc = rcfg(16, 16, 4)
    g, e = b.adjoint(rc, torch.zeros((16, 16, 3), device="cuda"), sc.mats, mot)
    assert not g.any() and not e.any()
    with pytest.raises(rtb200.RtError):
        b.adjoint(rtb200.render_cfg(0, 16, 4), torch.zeros((0, 16, 3), device="cuda"))
