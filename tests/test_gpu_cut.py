"""GPU plane cut vs the oracle: identical vertex arrays and triangle arrays
(bit-exact), watertight halves, conserved volume."""
import numpy as np
import pytest

from conftest import box_mesh, box_with_cavity, l_shape, is_watertight, nested_tori
from cuacd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _check(ctx, oracle, v, t, plane):
    g = ctx.plane_cut(v, t, plane)
    o = oracle.plane_cut(v, t, plane)
    for a, b in zip(g, o[:4]):
        np.testing.assert_array_equal(a, b)
    return g, o[4]


@pytest.mark.parametrize("plane", [(0, 0, 1, -0.5), (0, 0, 1, -0.25), (1, 0, 0, -0.5), (0, 1, 0, -0.7),
                                   (0.6, 0.48, 0.64, -0.9)])
def test_cube(ctx, oracle, plane):
    v, t = box_mesh([0, 0, 0], [1, 1, 1])
    (pv, pt, nv, nt), info = _check(ctx, oracle, v, t, plane)
    assert is_watertight(pt) and is_watertight(nt)


def test_plane_through_vertices_and_faces(ctx, oracle):
    v, t = box_mesh([0, 0, 0], [1, 1, 1])
    _check(ctx, oracle, v, t, (1, 0, 0, 0))       # coplanar with a face
    _check(ctx, oracle, v, t, (1, 1, 0, -1))      # through an edge diagonal
    _check(ctx, oracle, v, t, (1, 0, 0, -2))      # misses the mesh


def test_lshape_and_disjoint(ctx, oracle):
    v, t = l_shape()
    _check(ctx, oracle, v, t, (0, 0, 1, -0.25))
    _check(ctx, oracle, v, t, (1, 0, 0, -1.5))
    a = box_mesh([0, 0, 0], [1, 1, 1]); b = box_mesh([3, 0, 0], [4, 1, 1])
    v = np.vstack([a[0], b[0]]); t = np.vstack([a[1], b[1] + 8])
    (pv, pt, nv, nt), info = _check(ctx, oracle, v, t, (1, 0, 0, -2))   # separates components, no crossing
    assert len(pt) == 12 and len(nt) == 12
    _check(ctx, oracle, v, t, (0, 0, 1, -0.5))                            # two loops


def test_candidate_mesh_planes(ctx, oracle):
    v, t = W.candidate_mesh()
    planes = list(oracle.concave_planes(v, t, 16, 0.005, 3.49)[:12])
    planes += [oracle.axis_plane(v, 3, i, 0.0125) for i in range(3)]
    total = oracle.mesh_volume(v, t)
    for p in planes:
        (pv, pt, nv, nt), info = _check(ctx, oracle, v, t, p)
        assert is_watertight(pt) and is_watertight(nt)
        assert abs(oracle.mesh_volume(pv, pt) + oracle.mesh_volume(nv, nt) - total) / total < 1e-6


def test_batch_meshes_random_planes(ctx, oracle):
    rng = np.random.default_rng(4)
    for v, t in W.batch_meshes(6, 500, 20000, seed=9):
        for _ in range(3):
            n = rng.standard_normal(3); n /= np.linalg.norm(n)
            p = (*n.astype(np.float32), np.float32(rng.uniform(-0.3, 0.3)))
            _check(ctx, oracle, v, t, p)


def test_nested_loops_and_holes(ctx, oracle):
    """Caps with holes and nesting (loop orientation, parent search, hole
    bridging): three concentric tori cut across their ring give six nested
    circles (annuli inside annuli); a box with an inverted inner box (a
    cavity) gives a square with a square hole."""
    v, t = nested_tori()
    for plane in [(0, 0, 1, -0.013), (0, 0, 1, 0.1), (0.08, 0.05, 0.9955, -0.02), (1, 0, 0, -0.05)]:
        n = np.asarray(plane[:3], np.float64)
        p = (*(n / np.linalg.norm(n)).astype(np.float32), np.float32(plane[3]))
        (pv, pt, nv_, nt), info = _check(ctx, oracle, v, t, p)
        assert is_watertight(pt) and is_watertight(nt)
    v, t = box_with_cavity()
    for plane in [(0, 0, 1, -0.5), (0, 1, 0, -0.45), (0.6, 0.48, 0.64, -0.9)]:
        (pv, pt, nv_, nt), info = _check(ctx, oracle, v, t, plane)
        assert is_watertight(pt) and is_watertight(nt)
