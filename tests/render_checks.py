"""Shared pieces of the path-loop parity tests: the oracle's render settings from the product's,
the camera record both sides use, and the statistical comparison of two independent Monte
Carlo estimates of one image.

The reference renders every sample from one std::mt19937 stream (src/main.cpp:333), which no
parallel renderer reproduces sample by sample, so images from different random streams are
compared as estimates: per pixel channel, the difference of the two means against three
standard errors of that difference, and the relative error of the image mean."""
import numpy as np

from oracle import OrcRenderCfg

# a scene of the reference's own test_traverse shapes seen from above the floor, so that most
# pixels see geometry and paths run several bounces
VIEW_SCN = "screen 96 72\ncamera 0 4 -9 lookat 0 0 4 60\n"


def orc_cfg_from(rc) -> OrcRenderCfg:
    o = OrcRenderCfg()
    for name, _ in OrcRenderCfg._fields_:
        val = getattr(rc, name)
        if hasattr(val, "__len__"):
            getattr(o, name)[:] = list(val)
        else:
            setattr(o, name, val)
    return o


def cam13_of(rc) -> np.ndarray:
    """pos, fwd, right, up, tan(fov_y / 2) of a render config (the reference's Camera fields)."""
    return np.array(list(rc.cam_pos) + list(rc.cam_fwd) + list(rc.cam_right) + list(rc.cam_up) + [rc.tan_half_fov_y],
                    np.float32)


def compare_estimates(a, a2, n_a, b, b2, n_b, tag, within=0.99, rel_mean=1e-3):
    """a, b: per-pixel means (H, W, 3); a2, b2: means of squares; n_a, n_b: samples per pixel.

    Passes when at least `within` of the pixel channels differ by at most 3 standard errors of
    the difference plus the rounding bound of a float sum of n non-negative samples
    (n * 2^-24 of the mean; it matters where every sample is the same value, e.g. a surface
    seen through a background whose blue channel is constant), and the image means differ by
    at most `rel_mean` relative. Returns (fraction within, relative mean error)."""
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    var_a = np.maximum(np.asarray(a2, np.float64) - a * a, 0.0)
    var_b = np.maximum(np.asarray(b2, np.float64) - b * b, 0.0)
    se = np.sqrt(var_a / n_a + var_b / n_b)
    float_sum = max(n_a, n_b) * 2.0 ** -24 * np.maximum(np.abs(a), np.abs(b))
    ok = np.abs(a - b) <= 3.0 * se + float_sum + 1e-7
    frac = float(ok.mean())
    rel = float(abs(a.mean() - b.mean()) / max(abs(b.mean()), 1e-12))
    assert frac >= within, f"{tag}: only {frac:.4f} of pixel channels within 3 SE (want >= {within})"
    assert rel <= rel_mean, f"{tag}: relative mean error {rel:.2e} (want <= {rel_mean:.0e})"
    return frac, rel


def env_map(h=32, w=64, seed=3):
    """A seeded smooth equirectangular RGB map (h rows of w texels)."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    base = np.stack([0.5 + 0.5 * np.sin(xx / 5.0), 0.5 + 0.5 * np.cos(yy / 3.0), np.full((h, w), 0.7)], axis=2)
    return (base * rng.uniform(0.5, 1.5, size=(h, w, 3))).astype(np.float32)
