"""Candidate evaluator (cut + volumes + hulls + Hausdorff + costs) vs the
oracle: integer results identical; volumes 1e-5 relative; Hausdorff 1e-5
absolute."""
import numpy as np
import pytest

from cuacd_b200 import workloads as W

pytestmark = pytest.mark.gpu
VOL_RTOL = 1e-5
HD_ATOL = 1e-5


def planes_for(oracle, v, t, n_edge, width=3):
    p = list(oracle.concave_planes(v, t, 16, 0.005, 3.49)[:n_edge])
    p += [oracle.axis_plane(v, width, i, 0.0125) for i in range(width)]
    return np.array(p, np.float32)


def _compare(g, o):
    assert g["ok"] == o["ok"]
    if not o["ok"]:
        return
    assert g["nv"] == o["nv"] and g["nt"] == o["nt"] and g["n_cap"] == o["n_cap"]
    assert g["hull_nv"] == o["hull_nv"] and g["hull_nt"] == o["hull_nt"]
    for s in range(2):
        assert abs(g["mesh_vol"][s] - o["mesh_vol"][s]) <= VOL_RTOL * o["mesh_vol"][s]
        assert abs(g["hull_vol"][s] - o["hull_vol"][s]) <= VOL_RTOL * o["hull_vol"][s]
        assert abs(g["hausdorff"][s] - o["hausdorff"][s]) < HD_ATOL
        assert abs(g["cost_full"][s] - o["cost_full"][s]) < 1e-4


def test_config3_candidates(ctx, oracle):
    v, t = W.candidate_mesh()
    planes = planes_for(oracle, v, t, 27)
    assert len(planes) == 30
    g = ctx.eval_candidates(v, t, planes)
    o = oracle.eval_candidates(v, t, planes, threads=8)
    assert all(r["err"] == 0 for r in g), [hex(r["err"]) for r in g]
    for a, b in zip(g, o):
        _compare(a, b)


def test_small_mesh_and_bad_planes(ctx, oracle):
    v, t = W.candidate_mesh(48, 16)
    planes = planes_for(oracle, v, t, 6)
    planes = np.vstack([planes, [[0, 0, 0, 0], [1, 0, 0, -5]]]).astype(np.float32)   # degenerate, missing
    g = ctx.eval_candidates(v, t, planes)
    o = oracle.eval_candidates(v, t, planes, threads=4)
    for a, b in zip(g[:-2], o[:-2]):
        _compare(a, b)
    assert g[-2]["ok"] == 0 and g[-1]["ok"] == 0


def test_rv_only(ctx, oracle):
    v, t = W.candidate_mesh(64, 24)
    planes = planes_for(oracle, v, t, 8)
    g = ctx.eval_candidates(v, t, planes, hausdorff=False)
    o = oracle.eval_candidates(v, t, planes, hausdorff=False)
    for a, b in zip(g, o):
        _compare(a, b)
        assert a["hausdorff"] == (0.0, 0.0)


def test_candidate_planes_bit_exact(ctx, oracle):
    for v, t in [W.candidate_mesh(), W.candidate_mesh(64, 24)] + W.batch_meshes(4, 500, 5000, seed=5):
        for K, width in ((16, 3), (32, 30), (4, 5)):
            conc, axis, valid = ctx.candidate_planes(v, t, K, 0.005, 3.49, width, 0.0125)
            ref = oracle.concave_planes(v, t, K, 0.005, 3.49)
            np.testing.assert_array_equal(conc, ref)
            for i in range(width):
                a = oracle.axis_plane(v, width, i, 0.0125)
                if a is None:
                    assert not valid[i]
                else:
                    np.testing.assert_array_equal(axis[i], a)
