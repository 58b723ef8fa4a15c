"""Small seeded scenes shared by the parity tests (sizes the oracle finishes in seconds)."""
import numpy as np

from rtb200 import scenes

TEST_TRAVERSE_SCN = ("box 0 0 5 1 1 1 q 0 0 0 1\n"
                     "box 0 0 12 1 1 1 q 0 0 0 1\n"
                     "sphere 0 5 0 2\n"
                     "box 0 -3 0 20 0.1 20 q 0 0 0 1\n")


def identical(n, seed=3):
    """n copies of one triangle: every Morton code equal, so the Morton split hands the whole
    range to the binned SAH (src/bvh/bvh_bfs.cpp:102-107)."""
    v, t = scenes.soup(1, seed=seed)
    return np.tile(v, (n, 1)), (t[None, 0, :] + 3 * np.arange(n, dtype=np.uint32)[:, None]).astype(np.uint32)


def planar(n, seed=4):
    """a soup flattened onto z = 0.5 (a zero-extent axis: the scene-size guard of
    src/bvh/bvh_morton.cpp:63-74 and the spatial-extent skip of bvh_sah.cpp:145-148)."""
    v, t = scenes.soup(n, seed=seed)
    v[:, 2] = 0.5
    v[:, 3:] = (0.0, 0.0, 1.0)
    return v, t


def big_and_small(n=3000, seed=5):
    """a few huge triangles over a soup of tiny ones: spatial splits and clipping."""
    v, t = scenes.soup(n, seed=seed)
    big, bt = scenes.soup(6, seed=seed + 1, lo=0.5, hi=0.9)
    return scenes.concat([(v, t), (big, bt)])[:2]


def cornell_ico(level=3):
    cv, ct, _ = scenes.cornell()
    iv, it = scenes.icosphere(level, radius=0.4, center=(0.0, -0.4, 0.2))
    return scenes.concat([(cv, ct), (iv, it)])[:2]


def scene_set(mesh_reader=None):
    s = {
        "one": scenes.soup(1, seed=11),
        "two": scenes.soup(2, seed=12),
        "seventeen": scenes.soup(17, seed=13),
        "identical17": identical(17),
        "identical100": identical(100),
        "planar500": planar(500),
        "soup2k": scenes.soup(2000, seed=1),
        "soup20k": scenes.soup(20480, seed=2),
        "ico4": scenes.icosphere(4),
        "cornell_ico": cornell_ico(),
        "big_small": big_and_small(),
    }
    if mesh_reader is not None:
        s["test_traverse"] = mesh_reader(TEST_TRAVERSE_SCN)
    return s
