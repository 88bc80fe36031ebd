"""The oracle against the reference's own GPU outputs on the same seeded
inputs: hull vertex sets (D&C and k-DOP paths), mesh volumes, plane-cut
topology and fragment volumes, sampled Hausdorff distances."""
import numpy as np
import pytest

import ref_gpu_cases as RC
from ref_gpu_cases import M, REF


@pytest.mark.parametrize("case", [c[0] for c in M.hull_cases()])
def test_hull_sets(oracle, case):
    clouds = dict(M.hull_cases())[case]
    ours = [oracle.hull(c) for c in clouds]
    RC.check_hull_sets(clouds, [set(o[0].tolist()) for o in ours], RC.ref_sets(f"hull_{case}"), oracle.quantize)
    rvol = REF[f"hull_{case}_vol"]
    for o, r in zip(ours, rvol):
        assert abs(o[2] - r) <= RC.VOL_RTOL * abs(o[2])


def test_kdop_sets(oracle):
    clouds = M.kdop_clouds()
    ours = [oracle.hull(c) for c in clouds]
    assert [set(o[0].tolist()) for o in ours] == RC.ref_sets("kdop")
    assert (REF["kdop_nvnterr"][:, 2] == 0).all()
    for o, r in zip(ours, REF["kdop_vol"]):
        assert abs(o[2] - r) <= RC.VOL_RTOL * abs(o[2])


def test_mesh_volume(oracle):
    for (v, t), r in zip(M.volume_meshes(), REF["mesh_volume"]):
        o = oracle.mesh_volume(v, t)
        assert abs(o - r) <= RC.VOL_RTOL * abs(o)


@pytest.mark.parametrize("k", [0, 1])
def test_plane_cut(oracle, k):
    v, t, planes = M.cut_cases()[k]
    for p, cnt, vol in zip(planes, REF[f"cut{k}_counts"], REF[f"cut{k}_vols"]):
        pv, pt, nv, nt, info = oracle.plane_cut(v, t, p)
        assert [len(pv), len(pt), len(nv), len(nt)] == cnt.tolist(), p
        for side, (a, b) in enumerate(((pv, pt), (nv, nt))):
            assert abs(oracle.mesh_volume(a, b) - vol[side]) <= RC.VOL_RTOL * abs(vol[side])


def test_hausdorff(oracle):
    for k, (v, t) in enumerate(M.hausdorff_meshes()):
        hv, ht = REF[f"hd{k}_hull_v"], REF[f"hd{k}_hull_t"]
        o = oracle.hausdorff(hv, ht, v, t, threads=8)
        assert abs(o - float(REF[f"hd{k}_dist"][0])) < RC.HD_ATOL, k
