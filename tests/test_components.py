"""CPU pins for the connected-components oracle: the reference's
tests/test_decompose_components.py cases, an independent graph library
(scipy), and the inner-shell rule of cuda/postprocess.cuh:449-495."""
import numpy as np
import pytest
from scipy.sparse import coo_matrix
from scipy.sparse.csgraph import connected_components

import components_cases as CC


def signed_volume(v, t):
    if len(t) == 0:
        return 0.0
    v = v.astype(np.float64)
    return float(np.sum(v[t[:, 0]] * np.cross(v[t[:, 1]], v[t[:, 2]]))) / 6.0


def test_single_cube(oracle):
    v, t = CC.cube()
    assert oracle.components(v, t) == []


def test_two_disjoint_cubes(oracle):
    cs = oracle.components(*CC.merge([CC.cube((0, 0, 0)), CC.cube((5, 0, 0))]))
    assert len(cs) == 2
    assert sorted(len(c[0]) for c in cs) == [8, 8]
    assert sorted(len(c[1]) for c in cs) == [12, 12]


def test_three_disjoint_tetrahedra(oracle):
    cs = oracle.components(*CC.merge([CC.tetrahedron((0, 0, 0)), CC.tetrahedron((10, 0, 0)),
                                      CC.tetrahedron((0, 10, 0))]))
    assert len(cs) == 3
    assert sorted(len(c[0]) for c in cs) == [4, 4, 4]
    assert sorted(len(c[1]) for c in cs) == [4, 4, 4]


def test_shared_vertices_stay_connected(oracle):
    assert oracle.components(*CC.shared_face_cubes()) == []


def test_volume_conservation(oracle):
    v, t = CC.merge([CC.cube((0, 0, 0), 2.0), CC.cube((10, 0, 0), 3.0)])
    cs = oracle.components(v, t)
    assert abs(sum(abs(signed_volume(c[0], c[1])) for c in cs) - abs(signed_volume(v, t))) < 1e-3
    assert abs(sum(c[2] for c in cs) - 35.0) < 1e-9


def test_33_cubes(oracle):
    cs = oracle.components(*CC.merge([CC.cube((3 * i, 0, 0)) for i in range(33)]))
    assert len(cs) == 33
    for cv, ct, vol in cs:
        assert abs(signed_volume(cv, ct) - 1.0) < 1e-6 and abs(vol - 1.0) < 1e-9
    # numbered by smallest vertex: the cubes' input order
    assert [float(c[0][0, 0]) for c in cs] == [3.0 * i - 0.5 for i in range(33)]


def test_inner_shells_dropped_only_when_mixed(oracle):
    v, t = CC.shells_with_cavities(5)
    cs = oracle.components(v, t)
    assert len(cs) == 6              # 6 outer shells; 3 cavities and the stray vertex dropped
    assert all(signed_volume(c[0], c[1]) > 0 for c in cs)
    allin = oracle.components(*CC.merge([CC.inverted(CC.cube((0, 0, 0))), CC.inverted(CC.cube((4, 0, 0)))]))
    assert len(allin) == 2           # all inner: all kept


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_membership_matches_graph_library(oracle, seed):
    v, t = CC.shuffled(CC.many_boxes(60, seed), seed + 10)
    cs = oracle.components(v, t)
    n = len(v)
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]]])
    g = coo_matrix((np.ones(len(e)), (e[:, 0], e[:, 1])), shape=(n, n))
    k, lab = connected_components(g, directed=False)
    assert k == len(cs) == 60
    # component order = order of smallest vertex; vertex and triangle order = input order
    first = {}
    for i in range(n):
        first.setdefault(lab[i], i)
    order = sorted(first, key=lambda c: first[c])
    for c, (cv, ct, _) in zip(order, cs):
        idx = np.nonzero(lab == c)[0]
        np.testing.assert_array_equal(cv, v[idx])
        remap = np.full(n, -1)
        remap[idx] = np.arange(len(idx))
        np.testing.assert_array_equal(ct, remap[t[lab[t[:, 0]] == c]])
