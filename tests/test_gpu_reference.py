"""This library's CUDA path against the reference's own GPU outputs
(tests/golden/ref_gpu.npz) on the same seeded inputs: hull vertex sets and
counts, k-DOP hulls, mesh volumes, plane-cut topology and fragment volumes,
sampled Hausdorff distances, and the lookahead search's part count against
the reference's search with the same settings (north-star acceptance: at
most 10 % more parts, every part below tau)."""
import numpy as np
import pytest

import ref_gpu_cases as RC
from conftest import is_watertight
from ref_gpu_cases import M, REF

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", [c[0] for c in M.hull_cases()])
def test_hull_sets(ctx, oracle, case):
    clouds = dict(M.hull_cases())[case]
    meshes = ctx.batch_hull_dandc_mesh(clouds)
    ours = [set(M.index_set(c, hv).tolist()) for c, (hv, _, _) in zip(clouds, meshes)]
    ref = RC.ref_sets(f"hull_{case}")
    bad = RC.check_hull_sets(clouds, ours, ref, oracle.quantize)
    counts = REF[f"hull_{case}_nvnterr"]
    for i, ((hv, ht, vol), (rnv, rnt, rerr)) in enumerate(zip(meshes, counts)):
        if i not in bad:
            assert (len(hv), len(ht)) == (rnv, rnt), i
        assert abs(vol - REF[f"hull_{case}_vol"][i]) <= RC.VOL_RTOL * abs(vol) + 1e-7
    vols, errs = ctx.batch_hull_volume(clouds)
    assert not errs.any()


def test_kdop(ctx):
    clouds = M.kdop_clouds()
    meshes = ctx.batch_kdop_hull_mesh(clouds)
    assert [set(M.index_set(c, hv).tolist()) for c, (hv, _, _) in zip(clouds, meshes)] == RC.ref_sets("kdop")
    for (hv, ht, vol), (rnv, rnt, _), rvol in zip(meshes, REF["kdop_nvnterr"], REF["kdop_vol"]):
        assert (len(hv), len(ht)) == (rnv, rnt)
        assert abs(vol - rvol) <= RC.VOL_RTOL * abs(rvol)


def test_mesh_volume(ctx):
    ms = M.volume_meshes()
    g = ctx.batch_mesh_volume([m[0] for m in ms], [m[1] for m in ms])
    assert np.all(np.abs(g - REF["mesh_volume"]) <= RC.VOL_RTOL * np.abs(REF["mesh_volume"]))


@pytest.mark.parametrize("k", [0, 1])
def test_plane_cut(ctx, k):
    v, t, planes = M.cut_cases()[k]
    for p, cnt, vol in zip(planes, REF[f"cut{k}_counts"], REF[f"cut{k}_vols"]):
        pv, pt, nv, nt = ctx.plane_cut(v, t, p)
        assert [len(pv), len(pt), len(nv), len(nt)] == cnt.tolist(), p
        for side, (a, b) in enumerate(((pv, pt), (nv, nt))):
            assert is_watertight(b)
            got = ctx.batch_mesh_volume([a], [b])[0]
            assert abs(got - vol[side]) <= RC.VOL_RTOL * abs(vol[side]) + 1e-7


def test_hausdorff(ctx):
    for k, (v, t) in enumerate(M.hausdorff_meshes()):
        g = ctx.hausdorff(REF[f"hd{k}_hull_v"], REF[f"hd{k}_hull_t"], v, t)
        assert abs(g - float(REF[f"hd{k}_dist"][0])) < RC.HD_ATOL, k


@pytest.mark.parametrize("k", [0, 1])
def test_lookahead_part_count(ctx, k):
    v, t = M.lookahead_meshes()[k]
    parts = ctx.lookahead_decompose(v, t, **M.LOOKAHEAD_KW)
    n_ref = len(REF[f"la{k}_parts"])
    assert len(parts) <= 1.1 * n_ref, (len(parts), n_ref)
    vol = ctx.batch_mesh_volume([p[0] for p in parts], [p[1] for p in parts])
    total = ctx.batch_mesh_volume([v], [t])[0]
    assert abs(vol.sum() - total) <= 1e-4 * total
    hv = ctx.batch_mesh_volume([p[2] for p in parts], [p[3] for p in parts])
    rv = 0.3 * np.cbrt(3.0 / (4.0 * np.pi) * np.maximum(hv.astype(np.float64) - vol, 0.0))
    assert rv.max() < M.LOOKAHEAD_KW["threshold"] + 1e-6, rv.max()


def _max_rv(parts):
    worst = 0.0
    for pv, pt, hv, ht in parts:
        gap = max(abs(M.vol64(hv, ht)) - abs(M.vol64(pv, pt)), 0.0) if len(ht) else 0.0
        worst = max(worst, 0.3 * np.cbrt(3.0 / (4.0 * np.pi) * gap))
    return worst


def test_config4_sample_searches_match_reference(ctx):
    """Config 4's 64-mesh sample (displaced spheres and unions of boxes,
    540-327,680 triangles) with config 4's settings, as one batched search:
    per mesh at most 10 % more parts than the reference's own search
    (tests/golden/ref_gpu_search.npz, recorded on a B200), every part at or
    below tau (north-star acceptance), and the same total."""
    import os
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_gpu_search.npz"))
    meshes = M.W.batch_meshes(512, 500, 200_000, seed=3, select={i for i in range(512) if i % 16 in (0, 5)})
    assert [len(t) for _, t in meshes] == d["tris"].tolist()
    kw = dict(M.LOOKAHEAD_KW)
    kw.pop("quick_depth")
    res = ctx.lookahead_decompose_batch(meshes, **kw)
    counts = np.array([len(p) for p in res])
    assert (counts <= 1.1 * d["parts"]).all(), (counts, d["parts"])
    assert abs(int(counts.sum()) - int(d["parts"].sum())) <= 0.1 * d["parts"].sum()
    for p in res:
        assert _max_rv(p) <= M.LOOKAHEAD_KW["threshold"] + 1e-6
