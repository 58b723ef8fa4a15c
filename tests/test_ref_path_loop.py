"""The path loop's restatement (oracle/rt_oracle.c) pinned to the reference's own src/main.cpp,
compiled in place into oracle/_ref/<variant>/libref.so by oracle/build_ref.sh through
oracle/ref_main_harness.cpp, and the product's scene settings pinned to the same code.

* Bit for bit: parseSceneConfig's screen size and camera (main.cpp:218-285) against
  rt_scene_config; makeCameraLookAt / makeCameraQuat (main.cpp:43-66) against rt_camera_lookat
  / rt_camera_quat; primaryRay (69-83), toWorld(sampleCosineHemisphere) (123-141) and
  IBL::sample (107-117) against the restatement's versions on random inputs.
* Statistically: the restatement's render (Philox stream per pixel) against the reference's own
  pixel loop and pathTrace (main.cpp:145-204, 339-365; a std::mt19937 per pixel) at 4096
  samples per pixel on reference-semantics scenes -- sky or IBL background, albedo 0.8, 8
  bounces, roulette after bounce 2 -- with >= 99 % of pixel channels within 3 standard errors
  and the image means within 1e-3 relative.

CPU only; skipped where oracle/_ref was not built."""
import os
import tempfile

import numpy as np
import pytest

import rtb200
from oracle import Reference
from render_checks import VIEW_SCN, cam13_of, compare_estimates, env_map, orc_cfg_from
from scenes_for_tests import TEST_TRAVERSE_SCN

pytestmark = pytest.mark.skipif(not Reference.available("hybrid"), reason="oracle/_ref not built")

SETTINGS = {
    "lookat": "screen 96 72\ncamera 0 4 -9 lookat 0 0 4 60\n",
    "lookat_default_fov": "screen 64 48\ncamera 1 2 3 lookat 0 0.5 0\n",
    "lookat_straight_down": "screen 32 32\ncamera 0 5 0 lookat 0 0 0 45\n",
    "quat": "screen 80 60\ncamera 0 1 6 1.2 q 0.1 0.2 0.05 0.97\n",
    "quat_unnormalised": "screen 40 30\ncamera -2 1 -3 0.8 q 0 1 0 1\n",
    "no_camera": "screen 20 10\nambient 0.1 0.2 0.3\n",
    "defaults": "# nothing\n",
}


@pytest.fixture(scope="module")
def ref():
    return Reference("hybrid")


def write_scn(d, text):
    p = os.path.join(d, "s.scn")
    with open(p, "w") as f:
        f.write(text)
    return p


@pytest.mark.parametrize("name", sorted(SETTINGS))
def test_scene_settings_match_reference(ref, name):
    with tempfile.TemporaryDirectory() as d:
        p = write_scn(d, SETTINGS[name])
        (W, H), cam, _, _ = ref.scene_config(p)
        rc, ibl = rtb200.scene_config(p)
    assert (rc.width, rc.height) == (W, H), name
    assert np.array_equal(cam13_of(rc).view(np.uint32), cam.view(np.uint32)), (name, cam13_of(rc), cam)
    assert ibl == ""


def test_cameras_match_reference(ref):
    rng = np.random.default_rng(17)
    for _ in range(200):
        pos = rng.uniform(-5, 5, 3).astype(np.float32)
        tgt = rng.uniform(-5, 5, 3).astype(np.float32)
        fov = float(np.float32(rng.uniform(10, 120)))
        rc = rtb200.render_cfg(8, 8, 1, lookat=(pos, tgt, fov))
        assert np.array_equal(cam13_of(rc).view(np.uint32), ref.camera_lookat(pos, tgt, fov).view(np.uint32))
        q = rng.normal(size=4).astype(np.float32)
        focal = float(np.float32(rng.uniform(0.3, 3.0)))
        rc = rtb200.render_cfg(8, 8, 1, quat=(pos, q, focal))
        assert np.array_equal(cam13_of(rc).view(np.uint32), ref.camera_quat(pos, q, focal).view(np.uint32))


def test_primary_rays_match_reference(ref, orc):
    rng = np.random.default_rng(18)
    for W, H, look in ((96, 72, ((0, 4, -9), (0, 0, 4), 60.0)), (17, 5, ((1, 2, 3), (0, 0.5, 0), 33.0))):
        rc = rtb200.render_cfg(W, H, 1, lookat=look)
        n = 20000
        px = rng.integers(0, W, n); py = rng.integers(0, H, n)
        jx = rng.random(n, dtype=np.float32); jy = rng.random(n, dtype=np.float32)
        got = orc.primary_rays(orc_cfg_from(rc), px, py, jx, jy)
        want = ref.primary_rays(cam13_of(rc), W, H, px, py, jx, jy)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_cosine_directions_match_reference(ref, orc):
    rng = np.random.default_rng(19)
    n = 50000
    u1 = rng.random(n, dtype=np.float32); u2 = rng.random(n, dtype=np.float32)
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    nrm[:8] = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0.9, 0.43588989, 0), (-0.9, 0, 0.43588989),
               (0.89999, 0.4359, 0)]
    u1[:4] = (0.0, 1.0 - 2.0 ** -24, 0.5, 1e-30)
    got = orc.cosine_dirs(u1, u2, nrm)
    want = ref.cosine_dirs(u1, u2, nrm)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_ibl_lookup_matches_reference(ref, orc):
    rng = np.random.default_rng(20)
    emap = env_map(24, 48, seed=4)
    d = rng.normal(size=(30000, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:6] = [(0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0), (0, 0, 1), (0, 0, -1)]
    assert np.array_equal(orc.ibl_lookup(emap, d).view(np.uint32), ref.ibl_lookup(emap, d).view(np.uint32))


@pytest.mark.parametrize("background", ["sky", "ibl"])
def test_restated_render_converges_to_reference(ref, orc, background):
    """4096 samples per pixel, 96 x 72, the reference's shading (sky or IBL, albedo 0.8, 8
    bounces, roulette after 2) over the reference's own bake of the scene."""
    spp = 4096
    emap = env_map(32, 64, seed=3) if background == "ibl" else None
    with tempfile.TemporaryDirectory() as d:
        p = write_scn(d, TEST_TRAVERSE_SCN + VIEW_SCN)
        v, t = ref.scene_geometry(p)
        baked = ref.bake(v, t)
        rc, _ = rtb200.scene_config(p, rtb200.render_cfg(1, 1, spp, seed=7, env_kind=2 if emap is not None else 0))
    threads = os.cpu_count() or 1
    m, m2 = ref.path_render(baked, cam13_of(rc), rc.width, rc.height, spp, max_bounce=8, seed=11, env_map=emap,
                            threads=threads)
    g, g2 = orc.render(baked, orc_cfg_from(rc), threads=threads, want_sq=True, env_map=emap)
    compare_estimates(g, g2, spp, m, m2, spp, f"restatement vs reference ({background})")
