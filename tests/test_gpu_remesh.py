"""Remesh front end on the GPU (Context.preprocess / gpu_preprocess):
vertices and triangles equal to the oracle's (oracle/remesh.py) value for
value, and the properties the reference's own tests check
(tests/test_preprocess.py there) -- every output passes the GPU mesh audit
(watertight, manifold, oriented, no degenerate triangle), the extent grows
by 2 (0.9 / R) margin, volume follows scale, a sphere keeps its volume at
R = 128, bad arguments are refused."""
import numpy as np
import pytest

from conftest import box_mesh
from cuacd_b200 import workloads as W
from oracle import remesh as RM

pytestmark = pytest.mark.gpu


def _volume(v, t):
    v = np.asarray(v, np.float64)
    return float(np.einsum("ij,ij->i", v[t[:, 0]], np.cross(v[t[:, 1]], v[t[:, 2]])).sum() / 6.0)


def _cases():
    v, t = box_mesh([0, 0, 0], [1, 1, 1])
    sv, st = W.candidate_mesh(16, 8, 0.3, seed=1)
    return [("cube", v, t), ("open cube", v, t[:10]), ("reversed", v, t[:, ::-1].copy()),
            ("doubled slab", np.vstack([v, v + np.float32([0, 0, 1e-4])]), np.vstack([t, t[:, ::-1] + 8])),
            ("flat triangle", np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]])),
            ("lumpy sphere", sv, st)]


@pytest.mark.parametrize("R", [8, 16, 32])
def test_matches_the_oracle(ctx, R):
    for name, v, t in _cases():
        gv, gt = ctx.preprocess(v, t, resolution=R)
        ov, ot = RM.remesh(v, t, R)
        np.testing.assert_array_equal(gv, ov, err_msg=name)
        np.testing.assert_array_equal(gt, ot, err_msg=name)


@pytest.mark.parametrize("R", [32, 64, 128])
def test_outputs_pass_the_audit(ctx, R):
    for name, v, t in _cases():
        gv, gt = ctx.preprocess(v, t, resolution=R)
        audit = ctx.check_mesh(gv, gt)
        assert len(gt) and audit["flags"] == 0, (name, audit)
        assert _volume(gv, gt) > 0, name


@pytest.mark.parametrize("R", [32, 64, 128])
def test_cube_extent_grows_by_the_shift(ctx, R):
    v, t = box_mesh([0, 0, 0], [1, 1, 1])
    gv, _ = ctx.preprocess(v, t, resolution=R)
    margin = 1.0 + 2.0 * 3.0 / R
    assert float(gv[:, 0].max() - gv[:, 0].min()) == pytest.approx(1.0 + 2.0 * (0.9 / R) * margin, rel=0.02)


def test_scale_translation_and_sphere(ctx):
    v, t = box_mesh([0, 0, 0], [1, 1, 1])
    small = _volume(*ctx.preprocess(v, t, resolution=32))
    big = _volume(*ctx.preprocess(v * 5 + np.float32([7, -3, 2]), t, resolution=32))
    assert big / small == pytest.approx(125.0, rel=1e-3)
    sv, st = W.icosphere(3)
    gv, gt = ctx.preprocess(sv, st, resolution=128)
    assert ctx.check_mesh(gv, gt)["flags"] == 0
    assert _volume(gv, gt) == pytest.approx(4.19, rel=0.15)


def test_bad_arguments(ctx):
    v, t = box_mesh([0, 0, 0], [1, 1, 1])
    for r in (48, 4):
        with pytest.raises(ValueError):
            ctx.preprocess(v, t, resolution=r)
    with pytest.raises(RuntimeError):
        ctx.preprocess(v, np.array([[0, 1, 8]]), resolution=16)          # index outside [0, nv)
    with pytest.raises(RuntimeError):
        ctx.preprocess(np.zeros((3, 3), np.float32), np.array([[0, 1, 2]]), resolution=16)   # no extent
    with pytest.raises(RuntimeError):
        ctx.preprocess(v, t, resolution=2048)
    bad = v.copy()
    bad[3, 1] = np.nan
    with pytest.raises(RuntimeError):
        ctx.preprocess(bad, t, resolution=16)                            # refused before any GPU work
