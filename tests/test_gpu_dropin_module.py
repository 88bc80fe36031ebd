"""The reference's own CPython module (csrc/module.c, unmodified) built
against this library's headers and linked to libcuacd_b200.so
(oracle/Makefile.ref: oracle/_ref/_gpu_dropin.so), driven with the
reference's argument formats (csrc/module.c:159-525): every call lands in
this library and agrees with this library's own Python API, preprocess
included (a bad resolution raises RuntimeError there, as the module maps
any non-zero return)."""
import importlib.machinery
import importlib.util
import os

import numpy as np
import pytest

import cuacd_b200
from cuacd_b200 import workloads as W

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PATH = os.path.join(ROOT, "oracle", "_ref", "_gpu_dropin.so")


@pytest.fixture(scope="module")
def g():
    if not os.path.exists(PATH):
        pytest.skip("oracle/_ref/_gpu_dropin.so not built (its recipe needs the reference tree)")
    loader = importlib.machinery.ExtensionFileLoader("_gpu", PATH)
    mod = importlib.util.module_from_spec(importlib.util.spec_from_loader("_gpu", loader))
    loader.exec_module(mod)
    mod.set_fatbin(b"")
    mod.init(0, 0)
    yield mod
    mod.destroy()


def _key_set(v):
    return {tuple(p) for p in np.asarray(v, np.float32).tolist()}


def test_hull_dandc_and_volume(g, ctx):
    clouds = W.hull_clouds(8, 1000, 0)
    n = len(clouds)
    packed = np.ascontiguousarray(np.concatenate(clouds), np.float32)
    off = np.arange(0, 1000 * n + 1, 1000, dtype=np.int32)
    mhv, mht = 1000, 1996
    ov = np.empty(n * mhv * 3, np.float32); ot = np.empty(n * mht * 3, np.int32)
    onv, ont, err = (np.empty(n, np.int32) for _ in range(3))
    g.hull_dandc(packed.ctypes.data, len(packed), off.ctypes.data, n, 1000, mhv, mht, ov.ctypes.data,
                 ot.ctypes.data, onv.ctypes.data, ont.ctypes.data, err.ctypes.data)
    ours = ctx.batch_hull_dandc_mesh(clouds)
    for i in range(n):
        assert err[i] == 0
        hv = ov[i * mhv * 3:(i * mhv + onv[i]) * 3].reshape(-1, 3)
        assert _key_set(hv) == _key_set(ours[i][0])
        assert ont[i] == len(ours[i][1])
    meshes = [W.candidate_mesh(64, 24), W.hausdorff_sphere(level=3)]
    vv = [np.ascontiguousarray(m[0], np.float32) for m in meshes]
    tt = [np.ascontiguousarray(m[1], np.int32) for m in meshes]
    allv, allt = np.concatenate(vv), np.concatenate(tt)
    voff = np.cumsum([0] + [len(x) for x in vv]).astype(np.int32)
    toff = np.cumsum([0] + [len(x) for x in tt]).astype(np.int32)
    vols = np.empty(2, np.float32)
    g.batch_mesh_volume(allv.ctypes.data, len(allv), allt.ctypes.data, len(allt), toff.ctypes.data,
                        voff.ctypes.data, 2, vols.ctypes.data)
    assert np.array_equal(vols, ctx.batch_mesh_volume(vv, tt))


def test_plane_cut_and_hausdorff(g, ctx):
    v, t = W.candidate_mesh(64, 24)
    v = np.ascontiguousarray(v, np.float32); t = np.ascontiguousarray(t, np.int32)
    vcap, tcap = len(v) + 2 * len(t), 3 * len(t) + 64
    pv, nvv = np.empty(vcap * 3, np.float32), np.empty(vcap * 3, np.float32)
    pt, ntt = np.empty(tcap * 3, np.int32), np.empty(tcap * 3, np.int32)
    plane = (0.3, -0.5, 0.8, 0.05)
    counts = g.test_plane_cut(v.ctypes.data, len(v), t.ctypes.data, len(t), *plane, pv.ctypes.data, vcap,
                              pt.ctypes.data, tcap, nvv.ctypes.data, vcap, ntt.ctypes.data, tcap)
    p_v, p_t, n_v, n_t = ctx.plane_cut(v, t, plane)
    assert tuple(counts) == (len(p_v), len(p_t), len(n_v), len(n_t))
    (hv, ht, _), = ctx.batch_hull_dandc_mesh([v])
    hv = np.ascontiguousarray(hv, np.float32); ht = np.ascontiguousarray(ht, np.int32)
    out = np.zeros(1, np.float32)
    g.test_hausdorff(hv.ctypes.data, len(hv), ht.ctypes.data, len(ht), v.ctypes.data, len(v), t.ctypes.data,
                     len(t), out.ctypes.data)
    assert abs(out[0] - ctx.hausdorff(hv, ht, v, t)) <= 1e-6


def test_lookahead_and_preprocess(g, ctx):
    v, t = W.candidate_mesh(64, 24)
    v = np.ascontiguousarray(v, np.float32); t = np.ascontiguousarray(t, np.int32)
    (hv, ht, _), = ctx.batch_hull_dandc_mesh([v])
    hv = np.ascontiguousarray(hv, np.float32); ht = np.ascontiguousarray(ht, np.int32)
    raw = g.lookahead_decompose(v.ctypes.data, len(v), t.ctypes.data, len(t), hv.ctypes.data, len(hv),
                                ht.ctypes.data, len(ht), 100, 30, 5, 0.05, 2, 0, 16, 0, 0,
                                n_concave_edges=16)
    ours = ctx.lookahead_decompose(v, t, width=30, width2=5, depth=2, threshold=0.05, n_concave_edges=16)
    assert len(raw) == len(ours)
    for r, (pv, pt, phv, pht) in zip(raw, ours):
        vb, tb, nv, nt = r[:4]
        assert (nv, nt) == (len(pv), len(pt))
        assert np.array_equal(np.frombuffer(vb, np.float32).reshape(nv, 3), pv)
    vb, tb, pnv, pnt = g.preprocess(v.ctypes.data, len(v), t.ctypes.data, len(t), 64)
    ov, ot = ctx.preprocess(v, t, resolution=64)
    assert (pnv, pnt) == (len(ov), len(ot)) and pnt > 0
    assert np.array_equal(np.frombuffer(vb, np.float32).reshape(pnv, 3), ov)
    assert np.array_equal(np.frombuffer(tb, np.int32).reshape(pnt, 3), ot)
    with pytest.raises(RuntimeError):
        g.preprocess(v.ctypes.data, len(v), t.ctypes.data, len(t), 48)
