"""ctypes binding for the CPU oracle (libcuacd_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline leg, always as the checker.  The product package
(cuacd_b200) never imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libcuacd_oracle.so")
_lib = None


def reference_tree():
    """Where the reference tree lies in this checkout's machine (the
    CUACD_REFERENCE_TREE variable, else its mount point), or None."""
    ref = os.environ.get("CUACD_REFERENCE_TREE", "/root/reference")
    return ref if os.path.exists(os.path.join(ref, "cuda", "mm.cu")) else None


def build():
    """Compile the oracle with its Makefile (gcc only), and the reference's
    own GPU path into oracle/_ref with Makefile.ref where the reference tree
    is present (it skips itself otherwise)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    ref = reference_tree()
    if ref:
        subprocess.run(["make", "-s", "-j8", "-C", _HERE, "-f", "Makefile.ref", f"REF={ref}"], check=True)


class CandResult(ctypes.Structure):
    _fields_ = [
        ("ok", ctypes.c_int),
        ("nv", ctypes.c_int * 2), ("nt", ctypes.c_int * 2),
        ("n_cap", ctypes.c_int),
        ("hull_nv", ctypes.c_int * 2), ("hull_nt", ctypes.c_int * 2),
        ("mesh_vol", ctypes.c_double * 2), ("hull_vol", ctypes.c_double * 2),
        ("hausdorff", ctypes.c_double * 2),
        ("cost_rv", ctypes.c_double * 2), ("cost_full", ctypes.c_double * 2),
        ("score_rv", ctypes.c_double), ("score_full", ctypes.c_double),
    ]


class CutInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "n_pos_tris", "n_neg_tris", "n_cap", "n_loops", "n_boundary",
        "cap_failed", "n_cross")]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        I = ctypes.c_int
        F = ctypes.c_float
        _lib.orc_mesh_signed_volume.restype = ctypes.c_double
        _lib.orc_mesh_signed_volume.argtypes = [P, I, P, I]
        _lib.orc_quantize.argtypes = [P, I, P]
        _lib.orc_hull.argtypes = [P, I, P, I, P, P, I, P, P]
        _lib.orc_plane_cut.argtypes = [P, I, P, I, F, F, F, F,
                                       P, I, P, I, P, I, P, I, P, P, P, P, P]
        _lib.orc_hd_sample_count.argtypes = [P, I, P, I, F, I, I]
        _lib.orc_hd_samples.argtypes = [P, I, P, I, F, I, I, P, I]
        _lib.orc_hausdorff.restype = ctypes.c_double
        _lib.orc_hausdorff.argtypes = [P, I, P, I, P, I, P, I, F, I, I, I]
        _lib.orc_concave_planes.argtypes = [P, I, P, I, I, F, F, P]
        _lib.orc_axis_plane.argtypes = [P, I, I, I, F, P]
        _lib.orc_eval_candidates.argtypes = [P, I, P, I, P, I, I, F, I, I, I, P]
        _lib.orc_components.argtypes = [P, I, P, I, I, I, I, P, P, P, P, P]
        _lib.orc_cost_rv.restype = ctypes.c_double
        _lib.orc_cost_rv.argtypes = [ctypes.c_double, ctypes.c_double]
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32).reshape(-1, 3)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32).reshape(-1, 3)


def mesh_volume(verts, tris):
    v, t = _f32(verts), _i32(tris)
    return abs(lib().orc_mesh_signed_volume(v.ctypes.data, len(v), t.ctypes.data, len(t)))


def quantize(pts):
    p = _f32(pts)
    q = np.empty((len(p), 3), dtype=np.int32)
    lib().orc_quantize(p.ctypes.data, len(p), q.ctypes.data)
    return q


def hull(pts):
    """Exact hull of the quantised points: (vertex input indices, triangles
    into that list, volume).  Canonical order."""
    p = _f32(pts)
    n = len(p)
    vidx = np.empty(max(n, 1), dtype=np.int32)
    tcap = max(2 * n, 8)
    tris = np.empty((tcap, 3), dtype=np.int32)
    nv, nt = ctypes.c_int(0), ctypes.c_int(0)
    vol = ctypes.c_double(0)
    rc = lib().orc_hull(p.ctypes.data, n, vidx.ctypes.data, len(vidx), ctypes.byref(nv),
                        tris.ctypes.data, tcap, ctypes.byref(nt), ctypes.byref(vol))
    if rc < 0:
        raise RuntimeError("oracle hull capacity overflow")
    return vidx[:nv.value].copy(), tris[:nt.value].copy(), vol.value


def plane_cut(verts, tris, plane):
    v, t = _f32(verts), _i32(tris)
    cv, ct = 2 * len(v) + 16, 3 * len(t) + 16
    pv = np.empty((cv, 3), np.float32); pt = np.empty((ct, 3), np.int32)
    nv_ = np.empty((cv, 3), np.float32); nt_ = np.empty((ct, 3), np.int32)
    c = [ctypes.c_int(0) for _ in range(4)]
    info = CutInfo()
    rc = lib().orc_plane_cut(v.ctypes.data, len(v), t.ctypes.data, len(t),
                             *[float(x) for x in plane],
                             pv.ctypes.data, cv, pt.ctypes.data, ct,
                             nv_.ctypes.data, cv, nt_.ctypes.data, ct,
                             *[ctypes.byref(x) for x in c], ctypes.byref(info))
    if rc:
        raise RuntimeError("oracle plane cut capacity overflow")
    a, b, d, e = [x.value for x in c]
    return (pv[:a].copy(), pt[:b].copy(), nv_[:d].copy(), nt_[:e].copy(),
            {f: getattr(info, f) for f, _ in CutInfo._fields_})


def hd_samples(verts, tris, resolution=2000.0, min_samples=1000, total=0):
    v, t = _f32(verts), _i32(tris)
    n = lib().orc_hd_sample_count(v.ctypes.data, len(v), t.ctypes.data, len(t),
                                  resolution, min_samples, total)
    out = np.empty((max(n, 1), 3), np.float32)
    lib().orc_hd_samples(v.ctypes.data, len(v), t.ctypes.data, len(t),
                         resolution, min_samples, total, out.ctypes.data, n)
    return out[:n]


def hd_sample_count(verts, tris, resolution=2000.0, min_samples=1000, total=0):
    """Samples the reference's rule draws on one surface (cuda/hausdorff.cuh:380-382)."""
    v, t = _f32(verts), _i32(tris)
    return int(lib().orc_hd_sample_count(v.ctypes.data, len(v), t.ctypes.data, len(t),
                                         resolution, min_samples, total))


def hausdorff(av, at, bv, bt, resolution=2000.0, min_samples=1000, total=0, threads=1):
    av, at, bv, bt = _f32(av), _i32(at), _f32(bv), _i32(bt)
    return lib().orc_hausdorff(av.ctypes.data, len(av), at.ctypes.data, len(at),
                               bv.ctypes.data, len(bv), bt.ctypes.data, len(bt),
                               resolution, min_samples, total, threads)


def concave_planes(verts, tris, n_concave_edges=32, eps=0.005, threshold=3.49):
    v, t = _f32(verts), _i32(tris)
    out = np.zeros((4 * max(n_concave_edges, 1), 4), np.float32)
    n = lib().orc_concave_planes(v.ctypes.data, len(v), t.ctypes.data, len(t),
                                 n_concave_edges, eps, threshold, out.ctypes.data)
    return out[:n].copy()


def axis_plane(verts, width, cut_idx, min_edge_dist):
    v = _f32(verts)
    out = np.zeros(4, np.float32)
    rc = lib().orc_axis_plane(v.ctypes.data, len(v), width, cut_idx, min_edge_dist, out.ctypes.data)
    return None if rc else out


def eval_candidates(verts, tris, planes, hausdorff=True, resolution=2000.0,
                    min_samples=1000, total=0, threads=1):
    v, t = _f32(verts), _i32(tris)
    p = np.ascontiguousarray(planes, dtype=np.float32).reshape(-1, 4)
    out = (CandResult * len(p))()
    lib().orc_eval_candidates(v.ctypes.data, len(v), t.ctypes.data, len(t),
                              p.ctypes.data, len(p), 1 if hausdorff else 0,
                              resolution, min_samples, total, threads,
                              ctypes.cast(out, ctypes.c_void_p))
    res = []
    for r in out:
        res.append({
            "ok": r.ok, "nv": tuple(r.nv), "nt": tuple(r.nt), "n_cap": r.n_cap,
            "hull_nv": tuple(r.hull_nv), "hull_nt": tuple(r.hull_nt),
            "mesh_vol": tuple(r.mesh_vol), "hull_vol": tuple(r.hull_vol),
            "hausdorff": tuple(r.hausdorff), "cost_rv": tuple(r.cost_rv),
            "cost_full": tuple(r.cost_full), "score_rv": r.score_rv,
            "score_full": r.score_full})
    return res


def components(verts, tris, max_comp=4096):
    """Connected components: list of (verts, tris, |volume|) in canonical
    order, or [] when the mesh is one component."""
    v, t = _f32(verts), _i32(tris)
    ov = np.empty((max(len(v), 1), 3), np.float32)
    ot = np.empty((max(len(t), 1), 3), np.int32)
    cnv = np.zeros(max_comp, np.int32)
    cnt = np.zeros(max_comp, np.int32)
    cvol = np.zeros(max_comp, np.float64)
    n = lib().orc_components(v.ctypes.data, len(v), t.ctypes.data, len(t), max_comp, len(ov), len(ot),
                             ov.ctypes.data, ot.ctypes.data, cnv.ctypes.data, cnt.ctypes.data,
                             cvol.ctypes.data)
    if n < 0:
        raise RuntimeError("oracle components capacity overflow")
    out, vo, to = [], 0, 0
    for c in range(n):
        out.append((ov[vo:vo + cnv[c]].copy(), ot[to:to + cnt[c]].copy(), float(cvol[c])))
        vo += cnv[c]
        to += cnt[c]
    return out


def mesh_audit(verts, tris):
    """Verdict bits of the reference's mesh audit (cuda/mesh_audit.cuh:92-157):
    1 a repeated-index or exactly zero-area triangle (FP32 cross product,
    no fused operations), 2 an index outside [0, nv) (that triangle is
    skipped), 4 an edge used by one triangle, 8 by more than two, 16 by two
    in the same direction."""
    v = np.asarray(verts, np.float32).reshape(-1, 3)
    t = np.asarray(tris, np.int64).reshape(-1, 3)
    nv = len(v)
    flags = 0
    bad = ((t < 0) | (t >= nv)).any(axis=1)
    if bad.any():
        flags |= 2
    t = t[~bad]
    if len(t) == 0:
        return flags
    a, b, c = t[:, 0], t[:, 1], t[:, 2]
    rep = (a == b) | (b == c) | (a == c)
    ab = (v[b] - v[a]).astype(np.float32)
    ac = (v[c] - v[a]).astype(np.float32)
    nx = ab[:, 1] * ac[:, 2] - ab[:, 2] * ac[:, 1]
    ny = ab[:, 2] * ac[:, 0] - ab[:, 0] * ac[:, 2]
    nz = ab[:, 0] * ac[:, 1] - ab[:, 1] * ac[:, 0]
    zero = (nx * nx + ny * ny + nz * nz) <= np.float32(0.0)
    if (rep | zero).any():
        flags |= 1
    e0 = np.concatenate([a, b, c])
    e1 = np.concatenate([b, c, a])
    lo, hi = np.minimum(e0, e1), np.maximum(e0, e1)
    key = lo * (1 << 32) + hi
    uk, inv = np.unique(key, return_inverse=True)
    tot = np.bincount(inv, minlength=len(uk))
    fwd = np.bincount(inv, weights=(e0 < e1).astype(np.int64), minlength=len(uk)).astype(np.int64)
    if (tot == 1).any():
        flags |= 4
    if (tot > 2).any():
        flags |= 8
    if ((tot == 2) & ((fwd == 2) | (fwd == 0))).any():
        flags |= 16
    return flags
