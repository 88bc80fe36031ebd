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


def _rv_costs(parts):
    out = []
    for v, t, hv, ht in parts:
        def vol(V, T):
            V = V.astype(np.float64)
            return abs(float(np.einsum("ij,ij->i", V[T[:, 0]], np.cross(V[T[:, 1]], V[T[:, 2]])).sum()) / 6.0)
        g = max(vol(hv, ht) - vol(v, t), 0.0)
        out.append(0.3 * np.cbrt(3.0 / (4.0 * np.pi) * g))
    return out


def _ridged(lvl, amp, seed):
    v, t = W.icosphere(lvl)
    v, t = W.displaced_sphere(v, t, amp, seed, n_terms=6, fmin=2.0, fmax=5.0, ridged=True)
    return W.normalize_extent(v).astype(np.float32), t


def test_pruned_search_quality(ctx, oracle):
    """Learned level-0 pruning (top 48 of each part's planes by the trained
    scorer, then the exact search expands its 8 best level-0 cuts): the parts
    stay watertight, keep the volume, end below tau, and their count stays
    within 10 % of the exact search's over three ridged meshes."""
    from cuacd_b200 import scorer as S
    rv = S.Scorer.load(ctx, S.RV_WEIGHTS_PATH)
    kw = dict(width=30, width2=5, depth=2, threshold=0.05, max_iters=100)
    meshes = [W.candidate_mesh(64, 24), _ridged(4, 0.35, 1), W.candidate_mesh(96, 32, 0.35, seed=5)]
    n_exact = n_pruned = 0
    for v, t in meshes:
        pe = ctx.lookahead_decompose(v, t, **kw)
        pp = ctx.lookahead_decompose(v, t, scorer=rv, top_k=48, beam=8, **kw)
        ranked, cut, expanded = ctx.last_prune_stats
        assert cut < 0.5 * ranked and expanded <= cut
        n_exact += len(pe)
        n_pruned += len(pp)
        total = oracle.mesh_volume(v, t)
        assert abs(sum(oracle.mesh_volume(pv, pt) for pv, pt, _, _ in pp) - total) / total < 1e-4
        assert all(is_watertight(pt) for _, pt, _, _ in pp)
        assert max(_rv_costs(pp)) < 0.05
    assert n_pruned <= 1.10 * n_exact, (n_pruned, n_exact)


def test_beam_only_search(ctx):
    """Exact beam (no scorer): only the 4 best level-0 cuts of each part are
    expanded; every part still ends below tau."""
    v, t = _ridged(4, 0.35, 1)
    pp = ctx.lookahead_decompose(v, t, width=30, width2=5, depth=2, threshold=0.05, beam=4)
    ranked, cut, expanded = ctx.last_prune_stats
    assert ranked == 0 and cut == 0 and expanded > 0
    assert max(_rv_costs(pp)) < 0.05


def test_merge_hulls_pass(ctx, oracle):
    """merge_hulls (cuda/postprocess_merge.cu): one greedy round of pairwise
    merges.  Fewer parts, the same total volume, every merged part below tau,
    and each merged part's hull is the exact hull of its vertices."""
    v, t = W.candidate_mesh(64, 24)
    kw = dict(width=30, width2=5, depth=2, threshold=0.05, n_concave_edges=16)
    plain = ctx.lookahead_decompose(v, t, **kw)
    merged = ctx.lookahead_decompose(v, t, merge_hulls=True, **kw)
    assert len(merged) < len(plain)
    total = oracle.mesh_volume(v, t)
    assert abs(sum(oracle.mesh_volume(pv, pt) for pv, pt, _, _ in merged) - total) / total < 1e-4
    plain_keys = {(len(pv), len(pt)) for pv, pt, _, _ in plain}
    n_new = 0
    for pv, pt, hv, ht in merged:
        assert is_watertight(pt)
        vi, tri, hvol = oracle.hull(pv)
        if (len(pv), len(pt)) in plain_keys:         # untouched part: its own exact hull
            np.testing.assert_array_equal(np.unique(hv, axis=0), np.unique(pv[vi], axis=0))
        else:
            # merged part: the hull of both parts' hull vertices (each found on
            # its own part's quantisation grid), so corners that only the
            # merged grid resolves may be missing; the volume agrees
            n_new += 1
            assert len(hv) > 0 and abs(oracle.mesh_volume(hv, ht) - hvol) <= 1e-3 * hvol
            assert max(_rv_costs([(pv, pt, hv, ht)])) < 0.05
    assert n_new == len(plain) - len(merged)


def test_merge_hulls_pairs_match_oracle(ctx, oracle):
    """Which pairs the merge-hulls pass merges, and the parts it makes,
    against the pass restated on the CPU (oracle/merge_ref.py) from the same
    search's parts before merging: same matched pairs in the same order, and
    each merged part is both meshes concatenated with the exact hull of both
    hulls' vertices.  A candidate whose cost lay within 1e-4 of tau would
    make the decision depend on the last bits of FP32 sums; none may occur
    here."""
    from oracle import merge_ref as MR
    kw = dict(width=30, width2=5, depth=2, threshold=0.05, n_concave_edges=16)
    n_merged = 0
    for v, t in (W.candidate_mesh(64, 24), W.candidate_mesh(96, 32, 0.35, seed=5)):
        plain = ctx.lookahead_decompose(v, t, **kw)
        merged = ctx.lookahead_decompose(v, t, merge_hulls=True, **kw)
        matches, costs = MR.merge_pass(plain, 0.05, oracle)
        assert all(abs(x - 0.05) > 1e-4 for x in costs.values())
        partner = {p1: p2 for p1, p2 in matches}
        dead = {p2 for _, p2 in matches}
        expect = []
        for i, p in enumerate(plain):
            if i in dead:
                continue
            if i in partner:
                a, b = p, plain[partner[i]]
                pts = np.concatenate([a[2], b[2]]).astype(np.float32)
                vidx, tris, _ = oracle.hull(pts)
                expect.append((np.concatenate([a[0], b[0]]), np.concatenate([a[1], b[1] + len(a[0])]),
                               pts[vidx], tris))
            else:
                expect.append(p)
        assert len(merged) == len(expect), (len(merged), len(expect), matches)
        for got, exp in zip(merged, expect):
            for x, y in zip(got, exp):
                np.testing.assert_array_equal(x, y)
        n_merged += len(matches)
    assert n_merged > 0
