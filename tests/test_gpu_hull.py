"""GPU hull parity against the oracle (bit-exact corner sets and triangles,
volume within 1e-5 relative)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, is_watertight
from cuacd_b200 import workloads as W

pytestmark = pytest.mark.gpu
VOL_RTOL = 1e-5


def _gpu_hulls(ctx, clouds):
    return ctx.batch_hull_dandc_mesh(clouds)


def _check_exact(oracle, clouds, gpu):
    for c, (hv, ht, vol) in zip(clouds, gpu):
        vidx, tris, ovol = oracle.hull(c)
        np.testing.assert_array_equal(hv, c[vidx])
        np.testing.assert_array_equal(ht, tris)
        if ovol > 0:
            assert abs(vol - ovol) / ovol < VOL_RTOL


def test_config1_clouds_exact(ctx, oracle):
    clouds = W.hull_clouds(256, 1000, 0)
    _check_exact(oracle, clouds, _gpu_hulls(ctx, clouds))


def test_golden_clouds_exact(ctx, oracle):
    g = np.load(os.path.join(GOLDEN, "hull_qhull.npz"))
    clouds = [g[f"pts_{i}"] for i in range(int(g["n"]))]
    gpu = _gpu_hulls(ctx, clouds)
    _check_exact(oracle, clouds, gpu)
    for i, (hv, ht, vol) in enumerate(gpu):
        idx = np.array([np.flatnonzero((clouds[i] == p).all(1))[0] for p in hv])
        assert np.array_equal(np.sort(idx), g[f"qhull_vertices_{i}"])


def test_known_answers(ctx):
    cube = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], np.float32)
    tet = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    (cv, ct, cvol), (tv, tt, tvol) = ctx.batch_hull_dandc_mesh([cube, tet])
    assert (len(cv), len(ct)) == (8, 12) and abs(cvol - 1) < 1e-6 and is_watertight(ct)
    assert (len(tv), len(tt)) == (4, 4) and abs(tvol - 1 / 6) < 1e-6
    vols, errs = ctx.batch_hull_volume([cube, tet])
    assert np.all(errs == 0) and abs(vols[0] - 1) < 1e-6


def test_degenerate_and_uneven(ctx, oracle):
    rng = np.random.default_rng(7)
    cube = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], np.float32)
    clouds = [
        np.zeros((3, 3), np.float32),                                     # n < 4
        np.concatenate([cube, rng.uniform(0.1, 0.9, (200, 3))]).astype(np.float32),
        np.concatenate([cube, cube, cube]).astype(np.float32),           # duplicates
        rng.uniform(-1, 1, (5, 3)).astype(np.float32),
        rng.standard_normal((3000, 3)).astype(np.float32),
        np.c_[rng.uniform(0, 1, (100, 2)), np.zeros(100)].astype(np.float32),  # flat
    ]
    gpu = _gpu_hulls(ctx, clouds)
    assert len(gpu[0][0]) == 0
    _check_exact(oracle, clouds[1:5], gpu[1:5])
    assert abs(gpu[5][2]) < 1e-6


def test_large_fragment_like(ctx, oracle):
    v, _ = W.candidate_mesh()
    (hv, ht, vol), = _gpu_hulls(ctx, [v])
    _check_exact(oracle, [v], [(hv, ht, vol)])
    assert is_watertight(ht)


def test_kdop_caps(ctx):
    v, _ = W.candidate_mesh(64, 20)
    (hv, ht, vol), = ctx.batch_kdop_hull_mesh([v])
    assert 0 < len(hv) <= 4096 and len(ht) == 2 * len(hv) - 4


def test_flat_leaves_in_face_plane(ctx, oracle):
    """A fragment cloud (210 points of a lookahead cut of the ridged sphere
    candidate_mesh(64, 24), with two axis-cut caps) whose BVH leaves lie flat
    in hull faces: the leaf bound must keep their points on the face, or the
    wrap loses them (the hull failed with an extraction error).  Also the
    same cloud shuffled and in a batch with others."""
    c = np.load(os.path.join(GOLDEN, "hull_flat_leaves.npy"))
    rng = np.random.default_rng(0)
    clouds = [c] + [c[rng.permutation(len(c))] for _ in range(3)] + W.hull_clouds(4, 1000, 0)
    gpu = _gpu_hulls(ctx, clouds)
    _check_exact(oracle, clouds, gpu)
    vol, err = ctx.batch_hull_volume(clouds)
    assert not err.any()


def test_duplicated_extreme_point(ctx, oracle):
    """Two part clouds of a search (355 and 390 points) where 34 points
    quantise onto the lexicographic minimum, so the first seed's contact set
    is more than 24 points on one line: the seed must wrap again instead of
    taking them for a face (the hull came out empty, with no error)."""
    g = np.load(os.path.join(GOLDEN, "hull_dup_corner.npz"))
    clouds = [g["c0"], g["c1"]]
    _check_exact(oracle, clouds, _gpu_hulls(ctx, clouds))


def test_hull_above_65536_vertices(ctx):
    """A convex cloud whose hull has more than 65,536 vertices (the 163,842
    vertices of a level-7 icosphere: 79,206 on the hull grid), directly and
    as a fragment of the evaluator: the same vertex sets and sizes as the
    oracle (tests/golden/hull_big.npz, made by make_big_hull.py), never a
    truncated hull."""
    d = np.load(os.path.join(GOLDEN, "hull_big.npz"))
    v, t = W.icosphere(7)
    v = v.astype(np.float32)
    (hv, ht, vol), = ctx.batch_hull_dandc_mesh([v])
    first = {}
    for i, p in enumerate(map(tuple, v.tolist())):
        first.setdefault(p, i)
    idx = np.sort(np.array([first[tuple(p)] for p in hv.tolist()], np.int32))
    assert len(idx) > 65536
    np.testing.assert_array_equal(idx, np.sort(d["ico7_idx"]))
    assert len(ht) == 2 * len(hv) - 4
    r = ctx.eval_candidates(v, t, d["cut_plane"], hausdorff=False)[0]
    assert r["err"] == 0 and r["ok"] == int(d["cut_ok"])
    assert tuple(r["nv"]) == tuple(d["cut_nv"]) and tuple(r["nt"]) == tuple(d["cut_nt"])
    assert tuple(r["hull_nv"]) == tuple(d["cut_hull_nv"]) and tuple(r["hull_nt"]) == tuple(d["cut_hull_nt"])
    assert max(r["hull_nv"]) > 65536
    for s in range(2):
        assert abs(r["hull_vol"][s] - d["cut_hull_vol"][s]) <= VOL_RTOL * d["cut_hull_vol"][s]
        assert abs(r["mesh_vol"][s] - d["cut_mesh_vol"][s]) <= VOL_RTOL * d["cut_mesh_vol"][s]
