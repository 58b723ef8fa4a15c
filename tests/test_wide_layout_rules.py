"""The 8-wide layout's rules on the host restatement (tests/test_gpu_wide.py compares the GPU
layout with it field by field): over oracle-built trees, every binary leaf is reachable from
the root exactly once, every decoded child box contains its exact box, and each node's
children occupy distinct slots. Runs on the CPU."""
import numpy as np
import pytest

from test_gpu_build import SCENES, orc_cfg
from test_gpu_wide import _dec, wide_restatement


def exact_child_boxes(nodes, w):
    """(wide node, slot) -> the exact box of the binary node placed there, matched by reference:
    a leaf by its triangle range, an inner child by its wide index."""
    leaf = nodes["is_leaf"].astype(bool)
    depth = np.zeros(nodes.shape[0], np.int64)
    for i in range(nodes.shape[0]):
        if not leaf[i]:
            depth[nodes["a"][i]] = depth[i] + 1
            depth[nodes["b"][i]] = depth[i] + 1
    flag = ~leaf & (depth % 3 == 0)
    wid = np.cumsum(flag) - flag
    by_leaf = {(int(nodes["a"][i]), int(nodes["b"][i])): i for i in np.nonzero(leaf)[0]}
    by_wide = {int(wid[i]): i for i in np.nonzero(flag)[0]}
    out = {}
    for k in range(w.shape[0]):
        imask = int(w[k]["meta"]) >> 24
        for c in range(8):
            if w[k]["cnt"][c] == 0:
                continue
            i = by_wide[int(w[k]["ref"][c])] if imask >> c & 1 else by_leaf[(int(w[k]["ref"][c]), int(w[k]["cnt"][c]))]
            out[(k, c)] = (nodes["bmin"][i][:3], nodes["bmax"][i][:3])
    return out


@pytest.mark.parametrize("scene,preset", [("soup2k", "lbvh63"), ("soup20k", "sah4"), ("ico4", "hybrid"),
                                          ("cornell_ico", "lbvh30")])
def test_wide_layout_reaches_every_leaf_with_conservative_boxes(orc, scene, preset):
    v, t = SCENES[scene]
    nodes = orc.build(v, t, orc_cfg(preset)).nodes
    w = wide_restatement(nodes)
    boxes = exact_child_boxes(nodes, w)
    if nodes["is_leaf"][0]:
        assert w.shape[0] == 0
        return
    # leaves of the binary tree, by their triangle range
    leaves = {(int(nodes["a"][i]), int(nodes["b"][i])) for i in np.nonzero(nodes["is_leaf"])[0] if nodes["b"][i] > 0}
    seen = []
    stack = [0]
    while stack:
        k = stack.pop()
        node = w[k]
        meta = int(node["meta"])
        e = [(meta >> (8 * a)) & 0xFF for a in range(3)]
        imask = meta >> 24
        for c in range(8):
            if node["cnt"][c] == 0:
                continue
            lo = [_dec(node["p"][a], int(node["qlo"][a][c]), 2.0 ** (e[a] - 127)) for a in range(3)]
            hi = [_dec(node["p"][a], int(node["qhi"][a][c]), 2.0 ** (e[a] - 127)) for a in range(3)]
            assert all(lo[a] <= hi[a] for a in range(3))
            exact = boxes[(k, c)]
            assert all(lo[a] <= exact[0][a] and hi[a] >= exact[1][a] for a in range(3)), (k, c)
            if imask >> c & 1:
                # (a wide child's own frame may reach outside this box: the boxes of a tree with
                # spatial splits need not nest, and the wide loop tests each level's boxes alone)
                stack.append(int(node["ref"][c]))
            else:
                seen.append((int(node["ref"][c]), int(node["cnt"][c])))
    assert sorted(seen) == sorted(leaves)
