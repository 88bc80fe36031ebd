"""GPU parity of the connected-components split (gpu_test_postprocess_dc)
against the oracle: identical components, vertices and triangles."""
import numpy as np
import pytest

import components_cases as CC
from cuacd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def expect(oracle, v, t):
    cs = oracle.components(v, t)
    return [(c[0], c[1]) for c in cs] if cs else [(v, t)]


def check(ctx, oracle, v, t):
    got = ctx.decompose_components(v, t)
    want = expect(oracle, v, t)
    assert len(got) == len(want)
    for (gv, gt), (wv, wt) in zip(got, want):
        np.testing.assert_array_equal(gv, wv)
        np.testing.assert_array_equal(gt, wt)
    return got


@pytest.mark.parametrize("case", CC.cases(), ids=lambda c: c[0])
def test_cases_bit_exact(ctx, oracle, case):
    _, v, t = case
    check(ctx, oracle, v, t)


def test_reference_counts(ctx):
    assert len(ctx.decompose_components(*CC.cube())) == 1
    got = ctx.decompose_components(*CC.merge([CC.cube((3 * i, 0, 0)) for i in range(33)]))
    assert len(got) == 33 and all(len(v) == 8 and len(t) == 12 for v, t in got)


def test_large_shuffled(ctx, oracle):
    v, t = CC.shuffled(CC.many_boxes(3000, 4, spacing=2.5), 11)
    assert len(check(ctx, oracle, v, t)) == 3000


def test_cut_islands(ctx, oracle):
    """Pieces a plane leaves on a ridged sphere, several of them islands."""
    v, t = W.candidate_mesh(64, 32, 0.35, seed=2)
    n_multi = 0
    for plane in ((1.0, 0.0, 0.0, 0.81), (1.0, 0.0, 0.0, -0.883), (0.0, 0.0, 1.0, -0.792),
                  (0.0, 0.0, 1.0, -0.6)):
        pv, pt, nv_, nt_, _ = oracle.plane_cut(v, t, plane)
        for mv, mt in ((pv, pt), (nv_, nt_)):
            if len(mt):
                n_multi += len(check(ctx, oracle, mv, mt)) > 1
    assert n_multi >= 3


def test_large_connected_unchanged(ctx):
    v, t = W.candidate_mesh(256, 80, 0.35, seed=2)
    got = ctx.decompose_components(v, t)
    assert len(got) == 1
    np.testing.assert_array_equal(got[0][0], v)
    np.testing.assert_array_equal(got[0][1], t)


def test_capacity_error(ctx):
    v, t = CC.merge([CC.cube((3 * i, 0, 0)) for i in range(5)])
    with pytest.raises(RuntimeError):
        ctx.decompose_components(v, t, max_comp=3)
