"""Host-side image and scene-settings code (CPU only): the Radiance RGBE .hdr writer and reader
that replace stb_image_write / stbi_loadf (src/main.cpp:96-104, 368-382), and the .scn settings
parser (parseSceneConfig, src/main.cpp:207-285)."""
import os

import numpy as np
import pytest

import rtb200


def rgbe_tolerance(img):
    # one shared exponent: each channel is within 2^-8 of the pixel's largest channel (truncation)
    return np.max(img, axis=2, keepdims=True) * (2.0 ** -7)


@pytest.mark.parametrize("w,h", [(37, 5), (7, 3), (256, 17)])
def test_hdr_round_trip(tmp_path, w, h):
    rng = np.random.default_rng(w * h)
    img = (np.exp(rng.uniform(-8, 8, size=(h, w, 3))) * (rng.random((h, w, 3)) > 0.1)).astype(np.float32)
    img[0, :4] = 0.0                  # zero pixels
    img[1, :] = img[1, 0]             # a run (RLE path)
    p = str(tmp_path / "a.hdr")
    rtb200.write_hdr(p, img)
    back = rtb200.read_hdr(p)
    assert back.shape == img.shape
    assert np.all(np.abs(back - img) <= rgbe_tolerance(img) + 1e-30)
    assert np.all(back <= img * (1 + 1e-6) + 1e-30)  # truncation never rounds up
    with open(p, "rb") as f:
        head = f.read(200)
    assert head.startswith(b"#?RADIANCE\n") and b"FORMAT=32-bit_rle_rgbe" in head and f"-Y {h} +X {w}".encode() in head


def test_hdr_flip_and_errors(tmp_path):
    img = np.arange(2 * 9 * 3, dtype=np.float32).reshape(2, 9, 3) + 1.0
    p = str(tmp_path / "f.hdr")
    rtb200.write_hdr(p, img, flip_y=True)
    back = rtb200.read_hdr(p)
    assert np.allclose(back[::-1], img, rtol=2 ** -7)
    with pytest.raises(rtb200.RtError, match="RT_E_IO"):
        rtb200.read_hdr(str(tmp_path / "missing.hdr"))
    bad = tmp_path / "bad.hdr"
    bad.write_bytes(b"P6\n1 1\n255\n\x00\x00\x00")
    with pytest.raises(rtb200.RtError, match="RT_E_FORMAT"):
        rtb200.read_hdr(str(bad))


def test_scene_config(tmp_path):
    p = tmp_path / "s.scn"
    p.write_text("# comment\nscreen 320 200\ncamera 1 2 3 lookat 0 0 0 45\nambient 0.2 0.3 0.4\n"
                 "ibl maps/sky.hdr\nsphere 0 0 0 1\n")
    c, ibl = rtb200.scene_config(str(p))
    assert (c.width, c.height) == (320, 200) and ibl == "maps/sky.hdr"
    ref = rtb200.render_cfg(1, 1, 1, lookat=((1, 2, 3), (0, 0, 0), 45.0))
    for f in ("cam_pos", "cam_fwd", "cam_right", "cam_up"):
        assert list(getattr(c, f)) == list(getattr(ref, f)), f
    assert c.tan_half_fov_y == ref.tan_half_fov_y
    q = tmp_path / "q.scn"
    q.write_text("camera 0 1 -6 1.5 q 0 0.1 0 0.995\n")
    c, ibl = rtb200.scene_config(str(q))
    refq = rtb200.render_cfg(1, 1, 1, quat=((0, 1, -6), (0.995, 0, 0.1, 0), 1.5))
    assert (c.width, c.height, ibl) == (800, 600, "")
    for f in ("cam_pos", "cam_fwd", "cam_right", "cam_up"):
        assert list(getattr(c, f)) == list(getattr(refq, f)), f
    # a missing file keeps the reference's defaults
    c, _ = rtb200.scene_config(str(tmp_path / "none.scn"))
    d = rtb200.render_cfg(1, 1, 1)
    assert (c.width, c.height) == (800, 600) and list(c.cam_pos) == list(d.cam_pos)
