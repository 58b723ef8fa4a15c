"""GPU adjoint (rt_adjoint, path-replay backpropagation) against
  * the oracle's FP64 adjoint (stored paths, explicit products) on a small case;
  * central finite differences of rt_render (h = 1e-3, the same counter-based random numbers
    in both perturbed renders) of an L2 image loss, on 64 random albedo parameters and the
    light's radiance, and on 16 at the differentiable-rendering workload's full size; every
    parameter within 1e-2 relative (plus the float-rounding bound of its difference quotient);
and the torch.autograd.Function harness (tests/diff_harness.py) end to end.
Per-triangle albedo in the forward render is checked against the oracle too."""
import numpy as np
import pytest
import torch

import rtb200
from diff_harness import DiffScene
from oracle import Baked
from rtb200 import scenes
from render_checks import orc_cfg_from
from test_gpu_render import compare

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


def fd_case(n_ico_tris=5120, w=96, h=96, spp=8, target_spp=None):
    sc, init, gt = scenes.diff_scene(n_ico_tris=n_ico_tris)
    ds = DiffScene(sc)
    rc = rcfg(w, h, spp, max_bounce=4)
    em = ds.emission()
    with torch.no_grad():
        target = ds.render(torch.from_numpy(gt).cuda(), em, rcfg(w, h, target_spp or 4 * spp, max_bounce=4, seed=77))
    return ds, rc, torch.from_numpy(init).cuda(), em, target


def l2(img, target):
    return ((img.double() - target.double()) ** 2).sum()


def central_difference(img_p, img_m, target, spp, hstep):
    """(L(p + h) - L(p - h)) / 2h of the L2 loss, from the two images, and the bound of its
    float rounding. The difference is summed as (I+ - I-)(I+ + I- - 2T) in double, so pixels the
    perturbation does not reach (bit-equal in both renders: the same random numbers, the same
    arithmetic) add nothing. In a pixel it does reach, each image is a float sum of spp samples
    whose rounding is at most spp * 2^-24 of its magnitude, so I+ - I- is off by at most twice
    that; the bound adds those errors up with their weights |I+ + I- - 2T|."""
    p, m, t = img_p.double(), img_m.double(), target.double()
    fd = ((p - m) * (p + m - 2.0 * t)).sum().item() / (2 * hstep)
    changed = p != m
    noise = (((p + m - 2.0 * t).abs() * 2.0 * spp * 2.0 ** -24 * torch.maximum(p.abs(), m.abs()))[changed]).sum().item()
    return fd, noise / (2 * hstep)


def check_fd(ds, rc, alb, em, target, n_picks, seed):
    """Central differences (h = 1e-3, correlated random numbers) against the adjoint on n_picks
    random albedo parameters of triangles the camera sees and on the light's radiance: every
    parameter within 1e-2 relative plus the rounding bound of its own difference quotient, and
    the median relative error below 1e-3."""
    a = alb.clone().requires_grad_(True)
    e = em.clone().requires_grad_(True)
    l2(ds.render(a, e, rc), target).backward()
    g_alb, g_em = a.grad.cpu().numpy(), e.grad.cpu().numpy()
    seen = np.flatnonzero(np.abs(g_alb).max(axis=1) > 1e-3 * np.abs(g_alb).max())
    rng = np.random.default_rng(seed)
    picks = [(int(t), int(c)) for t, c in zip(rng.choice(seen, n_picks, replace=False), rng.integers(0, 3, n_picks))]
    hstep = 1e-3
    rows = []
    with torch.no_grad():
        for t, c in picks:
            ap, am = alb.clone(), alb.clone()
            ap[t, c] += hstep; am[t, c] -= hstep
            fd, noise = central_difference(ds.render(ap, em, rc), ds.render(am, em, rc), target, rc.spp, hstep)
            rows.append((f"albedo[{t},{c}]", fd, float(g_alb[t, c]), noise))
        light = 5
        for c in range(3):
            ep, emn = em.clone(), em.clone()
            ep[light, c] += hstep; emn[light, c] -= hstep
            fd, noise = central_difference(ds.render(alb, ep, rc), ds.render(alb, emn, rc), target, rc.spp, hstep)
            rows.append((f"emission[{light},{c}]", fd, float(g_em[light, c]), noise))
    rel = np.array([abs(fd - g) / max(abs(fd), 1e-30) for _, fd, g, _ in rows])
    bad = [(name, fd, g, noise) for name, fd, g, noise in rows if abs(fd - g) > 1e-2 * abs(fd) + noise]
    assert not bad, f"parameters outside 1e-2 relative + rounding bound: {bad[:6]}"
    assert np.median(rel) < 1e-3, np.median(rel)
    return rel


def test_adjoint_matches_central_differences():
    ds, rc, alb, em, target = fd_case()
    check_fd(ds, rc, alb, em, target, 64, seed=12)


def test_adjoint_matches_central_differences_at_full_size():
    """The differentiable-rendering workload's own size: 50,000-triangle icosphere in the
    Cornell box, 512 x 512, 32 spp, depth 4, target rendered at 1024 spp from the ground-truth
    albedos; 16 random albedo parameters and the light's radiance."""
    ds, rc, alb, em, target = fd_case(n_ico_tris=50000, w=512, h=512, spp=32, target_spp=1024)
    check_fd(ds, rc, alb, em, target, 16, seed=13)


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
