"""GPU Hausdorff vs the FP64 oracle (same samples; 1e-5 absolute on meshes
normalised to extent ~2) and the reference's golden fixture rule."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, box_mesh
from cuacd_b200 import workloads as W

pytestmark = pytest.mark.gpu
HD_ATOL = 1e-5


def test_reference_fixture(ctx, oracle):
    d = np.load(os.path.join(GOLDEN, "hausdorff_ref.npz"))
    for i in range(int(d["n_pairs"])):
        args = (d[f"verts_a_{i}"], d[f"tris_a_{i}"], d[f"verts_b_{i}"], d[f"tris_b_{i}"])
        g = ctx.hausdorff(*args)
        o = oracle.hausdorff(*args)
        assert abs(g - o) < HD_ATOL, (i, g, o)
        ref = float(d[f"ref_{i}"])
        assert abs(g - ref) / ref < 0.15 or g <= ref * 1.01


def test_known(ctx):
    v, t = W.icosphere(3)
    assert ctx.hausdorff(v, t, v, t) < 1e-5
    a = box_mesh([-1, -1, -1], [1, 1, 1]); b = box_mesh([-0.5, -0.5, -0.5], [0.5, 0.5, 0.5])
    h = ctx.hausdorff(*a, *b)
    assert 0.4 < h < 1.2


def test_mesh_vs_hull(ctx, oracle):
    v, t = W.hausdorff_sphere(level=4)
    (hv, ht, _), = ctx.batch_hull_dandc_mesh([v])
    for total in (0, 200000):
        g = ctx.hausdorff(hv, ht, v, t, total=total)
        o = oracle.hausdorff(hv, ht, v, t, total=total, threads=8)
        assert abs(g - o) < HD_ATOL, (total, g, o)


def test_small_brute_sizes(ctx, oracle):
    """Tiny target meshes (single BVH leaf) and a tetrahedron."""
    tet_v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    tet_t = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.int32)
    v, t = W.icosphere(1)
    g = ctx.hausdorff(tet_v, tet_t, v, t)
    o = oracle.hausdorff(tet_v, tet_t, v, t)
    assert abs(g - o) < HD_ATOL


def test_batch_matches_single_pairs(ctx, oracle):
    """cuacd_hausdorff_batch: every pair of a mixed batch gets the distance
    the single-pair entry point gives it (same samples, exact maximum), and
    the oracle's within 1e-5; repeated identical pairs agree."""
    v, t = W.hausdorff_sphere(level=3)
    (hv, ht, _), = ctx.batch_hull_dandc_mesh([v])
    iv, it = W.icosphere(2)
    a = box_mesh([-1, -1, -1], [1, 1, 1]); b = box_mesh([-0.5, -0.5, -0.5], [0.5, 0.5, 0.5])
    cv, ct = W.candidate_mesh(32, 12, 0.35, seed=3)
    (chv, cht, _), = ctx.batch_hull_dandc_mesh([cv])
    pairs = [(hv, ht, v, t), (*a, *b), (iv.astype(np.float32), it, *a), (chv, cht, cv, ct)] + [(hv, ht, v, t)] * 5
    got = ctx.hausdorff_batch(pairs)
    for i, p in enumerate(pairs):
        single = ctx.hausdorff(*p)
        assert got[i] == np.float32(single), (i, got[i], single)
        assert abs(got[i] - oracle.hausdorff(*p)) < HD_ATOL, i
    assert np.all(got[4:] == got[0])
