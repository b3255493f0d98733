"""The compressed 8-wide traversal tree (rp_cuda_scene_export_wide): a structural and geometric
check of what the device built from the binary LBVH.

Every triangle sits in exactly one wide leaf, every node is reached exactly once from the root,
and each child slot's quantized planes p + q 2^(e-127) (exact in binary64) enclose the box of
everything beneath that child.  The walks' hits are pinned separately against the oracle's
brute-force scan (test_gpu_parity.py).
"""

import numpy as np
import pytest

from rypath_b200 import abi, renderer, scenes

pytestmark = pytest.mark.gpu


def decode(nodes):
    raw = np.ascontiguousarray(nodes)
    p = raw[:, 0:12].copy().view(np.float32).astype(np.float64)           # (N, 3)
    e = raw[:, 12:15].astype(np.int64) - 127                               # (N, 3)
    imask = raw[:, 15].astype(np.uint32)
    links = raw[:, 16:32].copy().view(np.uint32)                           # base, tri_base, leaf mask, unused
    q = raw[:, 32:80].reshape(-1, 6, 8).astype(np.float64)                 # lo.x lo.y lo.z hi.x hi.y hi.z x slot
    step = np.ldexp(1.0, e)                                                # (N, 3)
    lo = p[:, :, None] + q[:, 0:3, :] * step[:, :, None]
    hi = p[:, :, None] + q[:, 3:6, :] * step[:, :, None]
    return imask, links, lo, hi


def check_tree(scene):
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    n = scene.triangle_count
    nodes, tris = built.scene.export_wide(n)
    built.scene.close()
    ids = tris[:, 0, 3].copy().view(np.uint32)
    np.testing.assert_array_equal(np.sort(ids), np.arange(n, dtype=np.uint32))
    tri_lo = tris[:, :, :3].min(axis=1).astype(np.float64)
    tri_hi = tris[:, :, :3].max(axis=1).astype(np.float64)
    imask, links, lo, hi = decode(nodes)
    count = nodes.shape[0]
    seen_nodes = np.zeros(count, np.int32)
    seen_leaves = np.zeros(n, np.int32)

    def subtree(i):
        """(lo, hi) of everything beneath node i, checking each slot's enclosure on the way."""
        seen_nodes[i] += 1
        base, tri_base, lmask = int(links[i, 0]), int(links[i, 1]), int(links[i, 2])
        box_lo, box_hi = np.full(3, np.inf), np.full(3, -np.inf)
        inner = leaves = 0
        for k in range(8):
            if (imask[i] >> k) & 1:
                c_lo, c_hi = subtree(base + inner)
                inner += 1
            elif (lmask >> k) & 1:
                leaf = tri_base + leaves
                leaves += 1
                seen_leaves[leaf] += 1
                c_lo, c_hi = tri_lo[leaf], tri_hi[leaf]
            else:
                continue
            assert np.all(lo[i, :, k] <= c_lo) and np.all(hi[i, :, k] >= c_hi), (i, k)
            box_lo, box_hi = np.minimum(box_lo, c_lo), np.maximum(box_hi, c_hi)
        assert inner + leaves >= 2 or count == 1
        return box_lo, box_hi

    import sys
    sys.setrecursionlimit(10000)
    subtree(0)
    assert (seen_nodes == 1).all()
    assert (seen_leaves == 1).all()
    return count


def test_wide_tree_of_the_cornell_box():
    assert check_tree(scenes.cornell_box(8, 8, 1)) >= 1


def test_wide_tree_of_a_mixed_scene():
    scene = scenes.mixed_scene(8, 8, 1, 4, subdivisions=3, sphere_count=4)
    count = check_tree(scene)
    # an 8-wide tree over n leaves has at least (n - 1) / 7 nodes and far fewer than n - 1
    n = scene.triangle_count
    assert (n - 1) / 7 <= count < (n - 1) / 2
