"""lookahead_decompose on the GPU: the reference's structural pins
(tests/test_lookahead.py:124-231, tests/test_boundary_loops.py:23-47):
convex input stays one part; an L-shape splits into 2-10 watertight parts
whose volumes sum to the input's; every final part is below tau."""
import numpy as np
import pytest

from conftest import box_mesh, l_shape, is_watertight
from cuacd_b200 import workloads as W
import components_cases as CC

pytestmark = pytest.mark.gpu


def _costs(oracle, parts):
    out = []
    for v, t, hv, ht in parts:
        mv = oracle.mesh_volume(v, t)
        hvol = oracle.mesh_volume(hv, ht) if len(ht) else 0.0
        out.append(oracle.lib().orc_cost_rv(hvol, mv))
    return out


def test_cube_one_part(ctx):
    v, t = box_mesh([0, 0, 0], [1, 1, 1])
    parts = ctx.lookahead_decompose(v, t, width=12, width2=3, depth=2, n_concave_edges=4)
    assert len(parts) == 1


def test_lshape(ctx, oracle):
    v, t = l_shape()
    parts = ctx.lookahead_decompose(v, t, width=12, width2=3, depth=2, n_concave_edges=4, threshold=0.05)
    assert 2 <= len(parts) <= 10
    total = oracle.mesh_volume(v, t)
    s = 0.0
    for pv, pt, hv, ht in parts:
        assert is_watertight(pt)
        s += oracle.mesh_volume(pv, pt)
    assert abs(s - total) / total < 1e-4
    assert max(_costs(oracle, parts)) < 0.05


def test_components_split_first(ctx, oracle):
    """Disjoint convex shells come back as one part each, without cuts
    (per-iteration components pass, csrc/lookahead.c:329-347)."""
    v, t = CC.merge([CC.cube((3 * i, 0, 0)) for i in range(5)])
    parts = ctx.lookahead_decompose(v, t, width=12, width2=3, depth=2, n_concave_edges=4)
    assert len(parts) == 5
    for pv, pt, hv, ht in parts:
        assert len(pv) == 8 and len(pt) == 12
        assert abs(oracle.mesh_volume(pv, pt) - 1.0) < 1e-6


def test_displaced_sphere(ctx, oracle):
    v, t = W.candidate_mesh(64, 24)
    parts = ctx.lookahead_decompose(v, t, width=12, width2=3, depth=2, n_concave_edges=8,
                                    threshold=0.08, max_iters=30)
    assert len(parts) >= 2
    total = oracle.mesh_volume(v, t)
    s = sum(oracle.mesh_volume(pv, pt) for pv, pt, _, _ in parts)
    assert abs(s - total) / total < 1e-4
    for pv, pt, hv, ht in parts:
        assert is_watertight(pt)
        # each part's hull is the exact hull of its vertices
        vi, tri, hvol = oracle.hull(pv)
        np.testing.assert_array_equal(hv, pv[vi])
