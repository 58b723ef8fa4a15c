"""Generates the golden fixtures of tests/golden/ by running the reference itself
(oracle/_ref/<variant>/libref.so, compiled from the reference's own sources by
oracle/build_ref.sh). Run from the repository root:

    python tests/golden/make_golden.py

Each fixture holds the input geometry, the reference's baked .bvh arrays, and rays with the
reference's bvh::trace results, for small seeded scenes."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "ray-tracer_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
from rtb200 import scenes  # noqa: E402
from scenes_for_tests import TEST_TRAVERSE_SCN, big_and_small, identical  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def scene_list(ref):
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "t.scn")
        open(p, "w").write(TEST_TRAVERSE_SCN)
        tt = ref.scene_geometry(p)
    return {
        "soup300": scenes.soup(300, seed=101),
        "ico2": scenes.icosphere(2, seed=102),
        "test_traverse": tt,
        "identical40": identical(40, seed=103),
        "big_small": big_and_small(400, seed=104),
    }


def main():
    rng = np.random.default_rng(105)
    ref0 = oracle.Reference("hybrid")
    for name, (v, t) in scene_list(ref0).items():
        for variant in ("hybrid", "lbvh30", "sah4"):
            ref = oracle.Reference(variant)
            b = ref.bake(v, t)
            lo, hi = v[:, :3].min(0), v[:, :3].max(0)
            rays = scenes.incoherent_rays(2000, lo - 0.1, hi + 0.1, seed=int(rng.integers(1 << 30)))
            hit, out, tri = ref.trace(b, rays)
            codes, perm, sbox = ref.morton(v, t)
            np.savez_compressed(os.path.join(OUT, f"{name}_{variant}.npz"), verts=v, tris=t, nodes=b.nodes.view(np.uint8),
                                btris=b.tris, bverts=b.verts, rays=rays, hit=hit, out=out, tri=tri, codes=codes,
                                perm=perm, scene_box=sbox)
            print(name, variant, b.nodes.shape[0], "nodes", int(hit.sum()), "hits")


if __name__ == "__main__":
    with open(os.devnull, "w") as dn:
        # the reference prints progress lines from C; keep them off the terminal
        saved = os.dup(1)
        os.dup2(dn.fileno(), 1)
        try:
            main()
        finally:
            os.dup2(saved, 1)
