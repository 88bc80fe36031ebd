"""The lookahead search over a batch of meshes, its last-level branch and
bound, and the quick levels.

- A batch search (cuacd_lookahead_decompose_batch) shares its launches
  across meshes but decides per part, so every mesh must come back with
  exactly the parts of a search of that mesh alone (exact and pruned).
- Branch and bound (la_compute_best_ub + la_hull's rough-hull bound,
  cuda/la_expand.cu:380-457 in the reference) only drops items that cannot
  beat their cutting part's path bound: the chosen cuts, hence the parts,
  stay the same while fewer fragment hulls are built.
- quick_depth adds the reference's quick levels (cuda/la_refine.cu:52-351):
  the structural pins of the reference's lookahead tests still hold."""
import numpy as np
import pytest

from conftest import l_shape, is_watertight
from cuacd_b200 import workloads as W

pytestmark = pytest.mark.gpu
KW = dict(width=30, width2=5, depth=2, threshold=0.05, max_iters=100, n_concave_edges=16)


def _meshes():
    out = [W.candidate_mesh(64, 24), W.candidate_mesh(96, 32, 0.35, seed=5)]
    v, t = W.icosphere(3)
    v, t = W.displaced_sphere(v, t, 0.4, 3, n_terms=6, fmin=2.0, fmax=5.0, ridged=True)
    out.append((W.normalize_extent(v).astype(np.float32), t))
    out.append(tuple(np.asarray(x) for x in l_shape()))
    rng = np.random.default_rng(4)
    out.append(W.random_boxes_mesh(3, 2000, rng))
    return [(np.asarray(v, np.float32), np.asarray(t, np.int32)) for v, t in out]


def _same(a, b):
    assert len(a) == len(b), (len(a), len(b))
    for pa, pb in zip(a, b):
        for x, y in zip(pa, pb):
            assert x.shape == y.shape and np.array_equal(x, y)


def test_batch_equals_single_searches(ctx):
    meshes = _meshes()
    single = [ctx.lookahead_decompose(v, t, **KW) for v, t in meshes]
    batch = ctx.lookahead_decompose_batch(meshes, **KW)
    assert len(batch) == len(meshes)
    for a, b in zip(single, batch):
        _same(a, b)


def test_batch_equals_single_pruned(ctx):
    from cuacd_b200 import scorer as S
    meshes = _meshes()[:3]
    with S.Scorer.load(ctx, S.RV_WEIGHTS_PATH) as sc:
        single = [ctx.lookahead_decompose(v, t, **KW, scorer=sc, top_k=24, beam=4) for v, t in meshes]
        batch = ctx.lookahead_decompose_batch(meshes, **KW, scorer=sc, top_k=24, beam=4)
    for a, b in zip(single, batch):
        _same(a, b)


def test_branch_and_bound_keeps_cuts_and_saves_hulls(ctx):
    meshes = _meshes()[:3]
    with_bnb = ctx.lookahead_decompose_batch(meshes, **KW, branch_and_bound=True)
    st_on = ctx.last_search_stats
    without = ctx.lookahead_decompose_batch(meshes, **KW, branch_and_bound=False)
    st_off = ctx.last_search_stats
    for a, b in zip(with_bnb, without):
        _same(a, b)
    assert st_on[4] > 0, st_on                       # items cut off by the bound
    assert st_off[4] == 0
    assert st_on[3] < st_off[3], (st_on, st_off)      # fewer fragment hulls built


def test_quick_depth_structural(ctx, oracle):
    for depth in (1, 2):
        v, t = l_shape()
        parts = ctx.lookahead_decompose(v, t, width=12, width2=3, depth=depth, quick_depth=1,
                                        n_concave_edges=4, threshold=0.05)
        assert 2 <= len(parts) <= 12
        total = oracle.mesh_volume(v, t)
        s = 0.0
        for pv, pt, hv, ht in parts:
            assert is_watertight(pt)
            s += oracle.mesh_volume(pv, pt)
            hvol = oracle.mesh_volume(hv, ht)
            assert oracle.lib().orc_cost_rv(hvol, oracle.mesh_volume(pv, pt)) < 0.05
        assert abs(s - total) / total < 1e-4


def test_quick_levels_add_hulls(ctx):
    meshes = _meshes()[:2]
    ctx.lookahead_decompose_batch(meshes, **KW, quick_depth=0, branch_and_bound=False)
    st0 = ctx.last_search_stats
    parts = ctx.lookahead_decompose_batch(meshes, **KW, quick_depth=1, branch_and_bound=False)
    st1 = ctx.last_search_stats
    assert st1[3] > st0[3], (st0, st1)
    for p in parts:
        assert len(p) >= 1
        for pv, pt, hv, ht in p:
            assert is_watertight(pt)
