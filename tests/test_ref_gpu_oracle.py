"""The oracle against the reference's own GPU outputs on the same seeded
inputs: hull vertex sets (D&C and k-DOP paths), mesh volumes, plane-cut
topology and fragment volumes, sampled Hausdorff distances, concave-edge
planes (tests/golden/ref_gpu_concave.npz)."""
import functools
import os

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


CONCAVE = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_gpu_concave.npz"))


@functools.lru_cache(maxsize=1)
def _concave_cases():
    return {c[0]: c for c in M.concave_cases()}


@pytest.mark.parametrize("case", list(_concave_cases()))
def test_concave_planes_match_reference(oracle, case):
    """The planes the reference's own kernel (la_find_concave_edges,
    cuda/la_concave.cu:48-363) emitted for the case, recorded on a B200, as
    a multiset against the oracle's: the same number of planes, each oracle
    plane matched to its own reference plane within 1e-6 per coefficient
    (the reference computes them with fast-math FP32, so the last bits
    differ; its emission order is atomic, so only the multiset counts)."""
    name, v, t, ne = _concave_cases()[case]
    ref = CONCAVE[f"{name}_planes"]
    ours = oracle.concave_planes(v, t, ne, M.CONCAVE_KW["eps"], M.CONCAVE_KW["threshold"])
    assert len(ours) == len(ref)
    used = np.zeros(len(ref), bool)
    for p in ours:
        d = np.abs(ref - p).max(axis=1)
        d[used] = np.inf
        j = int(np.argmin(d))
        assert d[j] <= 1e-6, (case, p, ref[j])
        used[j] = True
