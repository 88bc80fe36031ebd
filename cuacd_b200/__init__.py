"""cuacd_b200 — B200 (sm_100a) engine for cuacd's lookahead candidate path.

`Context` mirrors `cuacd.Context` (cuacd/__init__.py:55-454 in the
reference): same constructor, method names, argument meaning, return types
and error behaviour (RuntimeError "cuacd error <code>: <message>").  Every
method runs hand-written CUDA kernels from libcuacd_b200.so through its C
ABI (include/cuacd_b200.h); there is no CPU fallback — importing this
package fails if the library is missing.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libcuacd_b200.so")

if not os.path.exists(_LIB_PATH):
    raise ImportError(
        f"cuacd_b200 native library is missing ({_LIB_PATH}); build it with "
        f"`python -c 'import cuacd_b200.build as b; b.build()'` (needs nvcc)")

_lib = ctypes.CDLL(_LIB_PATH)

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float


class CandResult(ctypes.Structure):
    """Mirror of cuacd_cand_result (include/cuacd_b200.h)."""
    _fields_ = [
        ("ok", _I), ("nv", _I * 2), ("nt", _I * 2), ("n_cap", _I),
        ("hull_nv", _I * 2), ("hull_nt", _I * 2),
        ("mesh_vol", _F * 2), ("hull_vol", _F * 2), ("hausdorff", _F * 2),
        ("cost_rv", _F * 2), ("cost_full", _F * 2),
        ("score_rv", _F), ("score_full", _F), ("err", _I),
    ]


class PartResult(ctypes.Structure):
    _fields_ = [
        ("verts", ctypes.POINTER(ctypes.c_float)), ("tris", ctypes.POINTER(ctypes.c_int)),
        ("nv", _I), ("nt", _I),
        ("hull_verts", ctypes.POINTER(ctypes.c_float)), ("hull_tris", ctypes.POINTER(ctypes.c_int)),
        ("hull_nv", _I), ("hull_nt", _I),
        ("mesh_vol", _F), ("hull_vol", _F), ("hausdorff", _F),
    ]


class GpuResult(ctypes.Structure):
    _fields_ = [("parts", ctypes.POINTER(PartResult)), ("nparts", _I)]


def _sig(name, res, args):
    fn = getattr(_lib, name)
    fn.restype = res
    fn.argtypes = args
    return fn


_sig("gpu_init", _I, [ctypes.POINTER(_P), _I, ctypes.c_size_t])
_sig("gpu_destroy", None, [_P])
_sig("gpu_last_error", ctypes.c_char_p, [_P])
_sig("gpu_heap_compact", _I, [_P])
_sig("gpu_pool_usage", ctypes.c_size_t, [_P])
_sig("gpu_heap_stats", _I, [_P, ctypes.POINTER(ctypes.c_ulonglong * 6)])
_sig("gpu_hull_dandc", _I, [_P, _P, _I, _P, _I, _I, _I, _I, _P, _P, _P, _P, _P])
_sig("gpu_kdop_hull", _I, [_P, _P, _I, _P, _I, _I, _I, _P, _P, _P, _P, _P, _P])
_sig("gpu_batch_mesh_volume", _I, [_P, _P, _I, _P, _I, _P, _P, _I, _P])
_sig("gpu_test_mesh_volume", _I, [_P, _P, _I, _P, _I, _P])
_sig("cuacd_launch_count", ctypes.c_ulonglong, [_P])

_OPTIONAL = {}


def _opt(name, res, args):
    """Entry points bound lazily (a missing symbol raises at call time)."""
    try:
        _OPTIONAL[name] = _sig(name, res, args)
    except AttributeError:
        _OPTIONAL[name] = None


_opt("gpu_test_hausdorff", _I, [_P, _P, _I, _P, _I, _P, _I, _P, _I, _P])
_opt("cuacd_hausdorff", _I, [_P, _P, _I, _P, _I, _P, _I, _P, _I, _F, _I, _I, _P])
_opt("cuacd_hausdorff_batch", _I, [_P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _F, _I, _I, _P])
_opt("cuacd_hausdorff_batch_device", _I, [_P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _F, _I, _I, _P, _P])
_opt("gpu_mesh_audit", _I, [_P, _P, _I, _P, _I, ctypes.POINTER(ctypes.c_uint)])
_opt("gpu_test_plane_cut", _I, [_P, _P, _I, _P, _I, _F, _F, _F, _F,
                                _P, _I, _P, _I, _P, _I, _P, _I, _P, _P, _P, _P])
_opt("gpu_test_warp_sort", _I, [_P, _P, _I, _P, _I])
_opt("gpu_test_postprocess_dc", _I, [_P, _P, _I, _P, _I, _I, _I, _I, _P, _P, _P, _P, _P])
_opt("cuacd_eval_candidates", _I, [_P, _P, _I, _P, _I, _P, _I, _I, _F, _I, _I, _P])
_opt("cuacd_eval_candidates_device", _I, [_P, _P, _I, _P, _I, _P, _I, _I, _F, _I, _I, _P, _P])
_opt("cuacd_hull_batch_device", _I, [_P, _P, _P, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P])
_opt("lookahead_decompose", _I, [_P, _P, _I, _P, _I, _P, _I, _P, _I,
                                 _I, _I, _I, _F, _I, _I, _I, _I, _I, _I, _I,
                                 _I, _F, _F, _I, _I, ctypes.POINTER(GpuResult)])
_opt("gpu_result_free", None, [ctypes.POINTER(GpuResult)])
_opt("cuacd_lookahead_trace", _I, [_P, _P, _P, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I,
                                   _I, _I, _I, _F, _I, _I, _I, _F, _F, _I, ctypes.POINTER(GpuResult)])
_opt("cuacd_lookahead_decompose_pruned", _I, [_P, _P, _I, _F, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I,
                                              _I, _I, _I, _F, _I, _I, _I, _I, _I, _I, _F, _F, _I,
                                              ctypes.POINTER(GpuResult)])
_opt("cuacd_lookahead_decompose_batch", _I, [_P, _I, _P, _P, _P, _P, _P, _P, _P, _P,
                                             _I, _I, _I, _F, _I, _I, _I, _I, _I, _I, _I, _F, _F, _I, _I, _I,
                                             _P, _I, _F, _I, _P, _P])
_opt("cuacd_hull_set_tuning", _I, [_P, _I, _I, _I])
_opt("cuacd_hull_get_tuning", _I, [_P, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)])
_opt("cuacd_hull_set_table_limit", _I, [_P, _I, _I])
_opt("cuacd_hull_get_table_limit", _I, [_P, _I, ctypes.POINTER(_I)])
_opt("cuacd_device_info", _I, [_P, ctypes.c_char_p, _I, ctypes.POINTER(_I)])
_opt("cuacd_candidate_planes", _I, [_P, _P, _I, _P, _I, _I, _F, _F, _I, _F, _P, _P, _P])
_opt("cuacd_profile_stages", _I, [_P, _I])
_opt("cuacd_stage_times", _I, [_P, _P])
_opt("cuacd_scorer_n_params", _I, [])
_opt("cuacd_scorer_n_features", _I, [])
_opt("cuacd_scorer_create", _I, [_P, ctypes.c_uint, ctypes.POINTER(_P)])
_opt("cuacd_scorer_free", None, [_P])
_opt("cuacd_scorer_set_params", _I, [_P, _P])
_opt("cuacd_scorer_get_params", _I, [_P, _P])
_opt("cuacd_scorer_set_normalizer", _I, [_P, _P, _P])
_opt("cuacd_scorer_get_normalizer", _I, [_P, _P, _P])
_opt("cuacd_candidate_features", _I, [_P, _P, _P, _I, _P, _I, _F, _P, _I, _P])
_opt("cuacd_scorer_grad", _I, [_P, _P, _P, _P, _I, _P, _P])
_opt("cuacd_scorer_train", _I, [_P, _P, _P, _P, _I, _I, _I, _F, _F, ctypes.c_uint, _P])
_opt("cuacd_scorer_predict", _I, [_P, _P, _P, _I, _P])
_opt("cuacd_scorer_gemm_counts", None, [ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_ulonglong)])
_opt("cuacd_eval_candidates_pruned_device", _I, [_P, _P, _P, _I, _P, _I, _F, _P, _I, _I, _F, _I, _I, _I, _F,
                                                 _P, _P, _P, _P, _P])
_opt("cuacd_eval_candidates_pruned", _I, [_P, _P, _P, _I, _P, _I, _F, _P, _I, _I, _F, _I, _I, _I, _F,
                                          _P, _P, _P, _P])
_opt("gpu_preprocess", _I, [_P, _P, _I, _P, _I, _I, ctypes.POINTER(ctypes.POINTER(ctypes.c_float)),
                            ctypes.POINTER(_I), ctypes.POINTER(ctypes.POINTER(ctypes.c_int)), ctypes.POINTER(_I)])
_opt("cuacd_remesh_case_table", None, [_P])
_libc_free = ctypes.CDLL(None).free          # gpu_preprocess's outputs come from malloc
_libc_free.argtypes = [_P]
_libc_free.restype = None


def _fn(name):
    f = _OPTIONAL.get(name) or getattr(_lib, name, None)
    if f is None:
        raise RuntimeError(f"cuacd error -1: {name} is not available in this build")
    return f


def native_library_path():
    return _LIB_PATH


# verdict bits of gpu_mesh_audit (cuda/mesh_audit.cuh:21-26 in the reference)
MAV_DEGEN_TRI, MAV_BAD_INDEX, MAV_OPEN_EDGE, MAV_NONMANIFOLD, MAV_FLIPPED = 1, 2, 4, 8, 16


def _as_f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _as_i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a):
    return ctypes.c_void_p(None if a is None else a.ctypes.data)


class Context:
    """GPU context (mirror of cuacd.Context, cuacd/__init__.py:55-118).

    Parameters
    ----------
    device : int
        CUDA device ordinal; -1 keeps the current device.
    pool_bytes : int
        Device pool size in bytes; 0 lets the pool grow on demand.
    """

    def __init__(self, device=-1, pool_bytes=0):
        h = ctypes.c_void_p()
        rc = _lib.gpu_init(ctypes.byref(h), int(device), int(pool_bytes))
        if rc != 0:
            raise RuntimeError(f"cuacd error {rc}: gpu_init failed")
        self._h = h
        self._alive = True
        # launch shapes tuned for this device by cuacd_b200.autotune, if stored
        from . import autotune
        autotune.apply_stored(self)

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "_alive", False):
            _lib.gpu_destroy(self._h)
            self._alive = False

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *args):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, rc):
        if rc != 0:
            msg = _lib.gpu_last_error(self._h)
            raise RuntimeError(f"cuacd error {rc}: {msg.decode() if msg else ''}")

    def heap_compact(self):
        """No-op kept for API compatibility (the pool is an arena)."""
        self._check(_lib.gpu_heap_compact(self._h))

    def pool_usage(self):
        """High-water mark of device pool bytes."""
        return int(_lib.gpu_pool_usage(self._h))

    def heap_stats(self):
        """(output_live, output_allocs, output_releases, scratch_live,
        scratch_allocs, scratch_releases)."""
        out = (ctypes.c_ulonglong * 6)()
        self._check(_lib.gpu_heap_stats(self._h, ctypes.byref(out)))
        return tuple(int(x) for x in out)

    def launch_count(self):
        return int(_lib.cuacd_launch_count(self._h))

    # -- front end: audit and remesh ----------------------------------------
    def check_mesh(self, verts, tris):
        """Topology audit on the GPU (cuacd/__init__.py:124-152): a dict of
        booleans and the raw verdict bitmask -- watertight (no edge used by
        one triangle), manifold (none used by more than two), oriented (no
        edge used twice in one direction, no degenerate triangle),
        needs_remesh (any flag), degenerate, bad_index, flags."""
        v = _as_f32(verts).reshape(-1, 3)
        t = _as_i32(tris).reshape(-1, 3)
        flags = ctypes.c_uint(0)
        self._check(_fn("gpu_mesh_audit")(self._h, _ptr(v), len(v), _ptr(t), len(t), ctypes.byref(flags)))
        f = int(flags.value)
        return {
            "watertight": not (f & MAV_OPEN_EDGE),
            "manifold": not (f & MAV_NONMANIFOLD),
            "oriented": not (f & (MAV_FLIPPED | MAV_DEGEN_TRI)),
            "needs_remesh": bool(f),
            "degenerate": bool(f & MAV_DEGEN_TRI),
            "bad_index": bool(f & MAV_BAD_INDEX),
            "flags": f,
        }

    def preprocess(self, verts, tris, resolution=64):
        """Remesh into a watertight, manifold, consistently oriented mesh
        (cuacd/__init__.py:158-180): the mesh is normalised into a padded
        grid of resolution^3 nodes (a power of two >= 8, at most 1,024), the
        distance to it within 3 cells is signed by a flood fill from the
        grid's boundary, moved out by 0.9 cells and contoured by marching
        cubes.  Returns (verts float32 (n, 3), tris int32 (m, 3))."""
        r = int(resolution)
        if r & (r - 1) or r < 8:
            raise ValueError("resolution must be a power of two >= 8")
        v = _as_f32(verts).reshape(-1, 3)
        t = _as_i32(tris).reshape(-1, 3)
        pv, pt = ctypes.POINTER(ctypes.c_float)(), ctypes.POINTER(ctypes.c_int)()
        nv, nt = ctypes.c_int(0), ctypes.c_int(0)
        rc = _fn("gpu_preprocess")(self._h, _ptr(v), len(v), _ptr(t), len(t), r, ctypes.byref(pv), ctypes.byref(nv),
                                   ctypes.byref(pt), ctypes.byref(nt))
        try:
            self._check(rc)
            out_v = np.ctypeslib.as_array(pv, (nv.value, 3)).copy() if nv.value else np.zeros((0, 3), np.float32)
            out_t = np.ctypeslib.as_array(pt, (nt.value, 3)).copy() if nt.value else np.zeros((0, 3), np.int32)
        finally:
            _libc_free(ctypes.cast(pv, ctypes.c_void_p))
            _libc_free(ctypes.cast(pt, ctypes.c_void_p))
        return out_v, out_t

    # -- hulls --------------------------------------------------------------
    @staticmethod
    def _pack(pts_list):
        arrs = [p if (type(p) is np.ndarray and p.dtype == np.float32 and p.ndim == 2 and p.shape[1] == 3)
                else np.asarray(p, dtype=np.float32).reshape(-1, 3) for p in pts_list]
        packed = np.concatenate(arrs, axis=0) if arrs else np.zeros((0, 3), np.float32)
        off = np.zeros(len(arrs) + 1, dtype=np.int32)
        np.cumsum([len(a) for a in arrs], out=off[1:])
        return arrs, packed, off

    def _hull(self, pts_list, max_hv=None, max_ht=None, meshes=True):
        arrs, packed, off = self._pack(pts_list)
        n = len(arrs)
        ns = [len(a) for a in arrs]
        max_pts = max(ns)
        max_hv = max_pts if max_hv is None else max_hv
        max_ht = max(max(2 * k - 4 for k in ns), 4) if max_ht is None else max_ht
        # volumes only: the hull meshes stay on the device (no copy back)
        ov = np.empty(n * max(max_hv, 1) * 3, np.float32) if meshes else None
        ot = np.empty(n * max(max_ht, 1) * 3, np.int32) if meshes else None
        onv = np.empty(n, np.int32)
        ont = np.empty(n, np.int32)
        vol = np.empty(n, np.float32)
        err = np.empty(n, np.int32)
        self._check(_lib.gpu_kdop_hull(self._h, _ptr(packed), int(off[-1]), _ptr(off), n,
                                       max_hv, max_ht, _ptr(ov), _ptr(ot), _ptr(onv), _ptr(ont),
                                       _ptr(vol), _ptr(err)))
        return ov, ot, onv, ont, vol, err, max_hv, max_ht

    def batch_hull_volume(self, pts_list, algo=2):
        """Convex hull volume per cloud -> (float32[n] volumes, int32[n] errors).
        `algo` is accepted for compatibility and ignored."""
        if len(pts_list) == 0:
            return np.empty(0, np.float32), np.empty(0, np.int32)
        _, _, onv, ont, vol, err, _, _ = self._hull(pts_list, meshes=False)
        vol = np.where((onv > 0) & (ont > 0), vol, 0.0).astype(np.float32)
        return vol, err

    def _hull_meshes(self, pts_list, max_hv=None, max_ht=None):
        if len(pts_list) == 0:
            return []
        ov, ot, onv, ont, vol, err, mhv, mht = self._hull(pts_list, max_hv, max_ht)
        out = []
        for i in range(len(pts_list)):
            nv, nt = int(onv[i]), int(ont[i])
            v = ov[i * mhv * 3: i * mhv * 3 + nv * 3].reshape(nv, 3).copy()
            t = ot[i * mht * 3: i * mht * 3 + nt * 3].reshape(nt, 3).copy()
            out.append((v, t, float(vol[i]) if nt > 0 else 0.0))
        return out

    def batch_hull_dandc_mesh(self, pts_list):
        """Exact hull mesh per cloud -> [(verts f32[nv,3], tris i32[nt,3], volume)].
        Bounds: nv <= n_pts, nt <= 2*n_pts - 4."""
        return self._hull_meshes(pts_list)

    def batch_kdop_hull_mesh(self, pts_list):
        """Hull mesh per cloud with the reference's fixed output caps
        (4096 vertices / 8192 triangles, cuacd/__init__.py:289-290)."""
        return self._hull_meshes(pts_list, 4096, 8192)

    # -- volumes -------------------------------------------------------------
    def batch_mesh_volume(self, verts_list, tris_list):
        """Volume of each watertight mesh -> float32[n]."""
        n = len(verts_list)
        if n == 0:
            return np.empty(0, np.float32)
        va = [_as_f32(v).reshape(-1, 3) for v in verts_list]
        ta = [_as_i32(t).reshape(-1, 3) for t in tris_list]
        allv = np.ascontiguousarray(np.concatenate(va, axis=0))
        allt = np.ascontiguousarray(np.concatenate(ta, axis=0))
        vo = np.zeros(n + 1, np.int32)
        to = np.zeros(n + 1, np.int32)
        for i in range(n):
            vo[i + 1] = vo[i] + len(va[i])
            to[i + 1] = to[i] + len(ta[i])
        out = np.empty(n, np.float32)
        self._check(_lib.gpu_batch_mesh_volume(self._h, _ptr(allv), int(vo[-1]), _ptr(allt), int(to[-1]),
                                               _ptr(to), _ptr(vo), n, _ptr(out)))
        return out

    # -- Hausdorff / plane cut ---------------------------------------------
    def hausdorff(self, a_verts, a_tris, b_verts, b_tris, resolution=2000.0, min_samples=1000, total=0):
        """Bidirectional sampled Hausdorff distance between two meshes."""
        av, at = _as_f32(a_verts).reshape(-1, 3), _as_i32(a_tris).reshape(-1, 3)
        bv, bt = _as_f32(b_verts).reshape(-1, 3), _as_i32(b_tris).reshape(-1, 3)
        out = np.zeros(1, np.float32)
        self._check(_fn("cuacd_hausdorff")(self._h, _ptr(av), len(av), _ptr(at), len(at),
                                           _ptr(bv), len(bv), _ptr(bt), len(bt),
                                           float(resolution), int(min_samples), int(total), _ptr(out)))
        return float(out[0])

    def hausdorff_batch(self, pairs, resolution=2000.0, min_samples=1000, total=0):
        """Sampled Hausdorff distance of each (a_verts, a_tris, b_verts, b_tris)
        pair, all pairs in one batch -> float32[n]."""
        n = len(pairs)
        if n == 0:
            return np.empty(0, np.float32)

        def pack(items):
            vs = [_as_f32(x[0]).reshape(-1, 3) for x in items]
            ts = [_as_i32(x[1]).reshape(-1, 3) for x in items]
            voff = np.zeros(n + 1, np.int32); np.cumsum([len(v) for v in vs], out=voff[1:])
            toff = np.zeros(n + 1, np.int32); np.cumsum([len(t) for t in ts], out=toff[1:])
            return (np.ascontiguousarray(np.concatenate(vs)), voff, np.ascontiguousarray(np.concatenate(ts)), toff)

        av, avo, at, ato = pack([(p[0], p[1]) for p in pairs])
        bv, bvo, bt, bto = pack([(p[2], p[3]) for p in pairs])
        out = np.zeros(n, np.float32)
        self._check(_fn("cuacd_hausdorff_batch")(self._h, n, _ptr(av), _ptr(avo), _ptr(at), _ptr(ato),
                                                 _ptr(bv), _ptr(bvo), _ptr(bt), _ptr(bto), float(resolution),
                                                 int(min_samples), int(total), _ptr(out)))
        return out

    def plane_cut(self, verts, tris, plane):
        """Cut a closed mesh by plane (a,b,c,d) -> (pos_v, pos_t, neg_v, neg_t)."""
        v, t = _as_f32(verts).reshape(-1, 3), _as_i32(tris).reshape(-1, 3)
        cv, ct = 2 * len(v) + 16, 3 * len(t) + 16
        pv = np.empty((cv, 3), np.float32); pt = np.empty((ct, 3), np.int32)
        nv_ = np.empty((cv, 3), np.float32); nt_ = np.empty((ct, 3), np.int32)
        c = [ctypes.c_int(0) for _ in range(4)]
        self._check(_fn("gpu_test_plane_cut")(self._h, _ptr(v), len(v), _ptr(t), len(t),
                                              *[float(x) for x in plane],
                                              _ptr(pv), cv, _ptr(pt), ct, _ptr(nv_), cv, _ptr(nt_), ct,
                                              *[ctypes.byref(x) for x in c]))
        a, b, d, e = [x.value for x in c]
        return pv[:a].copy(), pt[:b].copy(), nv_[:d].copy(), nt_[:e].copy()

    def decompose_components(self, verts, tris, max_comp=4096):
        """Split a mesh into its vertex-connected components -> list of
        (verts, tris).  Same entry point as the reference's
        ``_gpu.test_postprocess_dc`` (tests/test_decompose_components.py:82-112):
        components in order of their smallest vertex, inner shells dropped
        when outer shells exist, a connected mesh returned as one component."""
        v, t = _as_f32(verts).reshape(-1, 3), _as_i32(tris).reshape(-1, 3)
        nv, nt = len(v), len(t)
        max_comp = max(1, min(int(max_comp), max(nv, 1)))
        vcap, tcap = nv + 16, nt + 16
        ov = np.zeros((max_comp * vcap, 3), np.float32)
        ot = np.zeros((max_comp * tcap, 3), np.int32)
        cnv = np.zeros(max_comp, np.int32)
        cnt = np.zeros(max_comp, np.int32)
        n = ctypes.c_int(0)
        self._check(_fn("gpu_test_postprocess_dc")(self._h, _ptr(v), nv, _ptr(t), nt, max_comp, vcap, tcap,
                                                   _ptr(ov), _ptr(ot), _ptr(cnv), _ptr(cnt), ctypes.byref(n)))
        return [(ov[c * vcap:c * vcap + cnv[c]].copy(), ot[c * tcap:c * tcap + cnt[c]].copy())
                for c in range(n.value)]

    # -- candidate planes ----------------------------------------------------
    def candidate_planes(self, verts, tris, n_concave_edges=32, concave_eps=0.005, concave_threshold=3.49,
                         width=0, min_edge_dist=0.0125):
        """Concave-edge planes (la_concave.cu rule) followed by `width` axis
        cuts -> (float32[n,4] concave planes, float32[width,4] axis planes,
        bool[width] axis valid)."""
        v, t = _as_f32(verts).reshape(-1, 3), _as_i32(tris).reshape(-1, 3)
        out = np.zeros((4 * n_concave_edges + width + 1, 4), np.float32)
        nc = ctypes.c_int(0)
        valid = np.zeros(max(width, 1), np.int32)
        self._check(_fn("cuacd_candidate_planes")(self._h, _ptr(v), len(v), _ptr(t), len(t), int(n_concave_edges),
                                                  float(concave_eps), float(concave_threshold), int(width),
                                                  float(min_edge_dist), _ptr(out), ctypes.byref(nc), _ptr(valid)))
        k = nc.value
        return out[:k].copy(), out[k:k + width].copy(), valid[:width].astype(bool)

    # -- candidate evaluator -------------------------------------------------
    def eval_candidates(self, verts, tris, planes, hausdorff=True, resolution=2000.0,
                        min_samples=1000, total=0):
        """Evaluate candidate planes on one closed mesh (cut, volumes, hulls,
        Hausdorff, part costs).  Returns a list of dicts, one per plane."""
        v, t = _as_f32(verts).reshape(-1, 3), _as_i32(tris).reshape(-1, 3)
        p = _as_f32(planes).reshape(-1, 4)
        out = (CandResult * len(p))()
        self._check(_fn("cuacd_eval_candidates")(self._h, _ptr(v), len(v), _ptr(t), len(t), _ptr(p), len(p),
                                                 1 if hausdorff else 0, float(resolution), int(min_samples),
                                                 int(total), ctypes.cast(out, ctypes.c_void_p)))
        return [cand_to_dict(r) for r in out]

    # -- lookahead -----------------------------------------------------------
    def lookahead_decompose(self, verts, tris, *, max_iters=100, width=60, width2=5, threshold=0.05,
                            depth=2, quick_depth=0, max_n_cutting=16, verbose=0, debug=0,
                            decompose_components=False, no_decompose_components_per_iter=False,
                            n_concave_edges=32, concave_eps=0.005, concave_threshold=3.49,
                            concave_iters=10, merge_hulls=False, scorer=None, top_k=8, margin=0.0, beam=0):
        """Convex decomposition by lookahead tree search ->
        [(verts, tris, hull_verts, hull_tris)] (cuacd/__init__.py:367-454).

        With `scorer` (a cuacd_b200.scorer.Scorer), level 0 cuts only the
        top_k planes of each cutting part by predicted score (plus those
        within `margin` of the k-th); with `beam` > 0 only the `beam` level-0
        cuts of each part with the lowest exact cost are expanded further.
        `self.last_prune_stats` then holds (level-0 planes ranked, planes
        cut, level-0 cuts expanded)."""
        verts = _as_f32(verts).reshape(-1, 3)
        tris = _as_i32(tris).reshape(-1, 3)
        if width2 is None:
            width2 = width
        total_width = width + 4 * n_concave_edges
        if total_width >= 512:
            raise ValueError(f"width + 4*n_concave_edges must be < 512 (got {total_width})")
        hull = self.batch_hull_dandc_mesh([verts])[0]
        hv, ht = _as_f32(hull[0]), _as_i32(hull[1])
        res = GpuResult()
        if scorer is None and not beam:
            fn = _fn("lookahead_decompose")
            self._check(fn(self._h, _ptr(verts), len(verts), _ptr(tris), len(tris), _ptr(hv), len(hv), _ptr(ht),
                           len(ht), int(max_iters), int(width), int(width2), float(threshold), int(depth),
                           int(quick_depth), int(max_n_cutting), int(verbose), int(debug),
                           int(bool(decompose_components)), int(not no_decompose_components_per_iter),
                           int(n_concave_edges), float(concave_eps), float(concave_threshold), int(concave_iters),
                           int(bool(merge_hulls)), ctypes.byref(res)))
        else:
            st = (ctypes.c_ulonglong * 3)()
            fn = _fn("cuacd_lookahead_decompose_pruned")
            self._check(fn(self._h, scorer._h if scorer is not None else None, int(top_k), float(margin), int(beam),
                           ctypes.cast(st, ctypes.c_void_p),
                           _ptr(verts), len(verts), _ptr(tris), len(tris), _ptr(hv), len(hv), _ptr(ht), len(ht),
                           int(max_iters), int(width), int(width2), float(threshold), int(depth),
                           int(max_n_cutting), int(verbose), int(bool(decompose_components)),
                           int(not no_decompose_components_per_iter), int(n_concave_edges), float(concave_eps),
                           float(concave_threshold), int(concave_iters), ctypes.byref(res)))
            self.last_prune_stats = (int(st[0]), int(st[1]), int(st[2]))
        return _take_parts(res)

    def lookahead_decompose_batch(self, meshes, *, max_iters=100, width=60, width2=5, threshold=0.05,
                                  depth=2, quick_depth=0, max_n_cutting=16, verbose=0,
                                  decompose_components=False, no_decompose_components_per_iter=False,
                                  n_concave_edges=32, concave_eps=0.005, concave_threshold=3.49,
                                  concave_iters=10, merge_hulls=False, branch_and_bound=True,
                                  scorer=None, top_k=8, margin=0.0, beam=0):
        """lookahead_decompose of every (verts, tris) of `meshes` in one
        search whose levels share their launches -> one part list per mesh,
        each equal to what lookahead_decompose of that mesh alone returns
        (the same scorer / top_k / margin / beam pruning when given).
        `self.last_search_stats`: level-0 planes ranked, planes cut, level-0
        cuts expanded, fragment hulls built, items cut off by the
        branch-and-bound, iterations run."""
        if len(meshes) == 0:
            return []
        total_width = width + 4 * n_concave_edges
        if total_width >= 512:
            raise ValueError(f"width + 4*n_concave_edges must be < 512 (got {total_width})")
        vs = [_as_f32(v).reshape(-1, 3) for v, _ in meshes]
        ts = [_as_i32(t).reshape(-1, 3) for _, t in meshes]
        hulls = self.batch_hull_dandc_mesh(vs)
        hvs = [_as_f32(h[0]).reshape(-1, 3) for h in hulls]
        hts = [_as_i32(h[1]).reshape(-1, 3) for h in hulls]

        def pack(arrs, dtype):
            off = np.zeros(len(arrs) + 1, np.int32)
            np.cumsum([len(a) for a in arrs], out=off[1:])
            cat = np.ascontiguousarray(np.concatenate(arrs).astype(dtype, copy=False)) if arrs else np.zeros((0, 3), dtype)
            return cat, off

        V, Vo = pack(vs, np.float32)
        T, To = pack(ts, np.int32)
        HV, HVo = pack(hvs, np.float32)
        HT, HTo = pack(hts, np.int32)
        n = len(meshes)
        res = (GpuResult * n)()
        st = (ctypes.c_ulonglong * 8)()
        fn = _fn("cuacd_lookahead_decompose_batch")
        self._check(fn(self._h, n, _ptr(V), _ptr(Vo), _ptr(T), _ptr(To), _ptr(HV), _ptr(HVo), _ptr(HT), _ptr(HTo),
                       int(max_iters), int(width), int(width2), float(threshold), int(depth), int(quick_depth),
                       int(max_n_cutting), int(verbose), int(bool(decompose_components)),
                       int(not no_decompose_components_per_iter), int(n_concave_edges), float(concave_eps),
                       float(concave_threshold), int(concave_iters), int(bool(merge_hulls)),
                       int(bool(branch_and_bound)), scorer._h if scorer is not None else None, int(top_k),
                       float(margin), int(beam), ctypes.cast(st, ctypes.c_void_p),
                       ctypes.cast(res, ctypes.c_void_p)))
        self.last_search_stats = tuple(int(x) for x in st[:6])
        out = []
        try:
            for i in range(n):
                out.append(_take_parts(res[i], free=False))
        finally:
            for i in range(n):
                _fn("gpu_result_free")(ctypes.byref(res[i]))
        return out


def _take_parts(res, free=True):
    """Copy a gpu_result's parts into numpy arrays (and free it)."""
    out = []
    try:
        for i in range(res.nparts):
            p = res.parts[i]
            v = np.ctypeslib.as_array(p.verts, (p.nv * 3,)).reshape(p.nv, 3).copy() if p.nv else np.zeros((0, 3), np.float32)
            t = np.ctypeslib.as_array(p.tris, (p.nt * 3,)).reshape(p.nt, 3).copy() if p.nt else np.zeros((0, 3), np.int32)
            hv_ = np.ctypeslib.as_array(p.hull_verts, (p.hull_nv * 3,)).reshape(p.hull_nv, 3).copy() if p.hull_nv else np.zeros((0, 3), np.float32)
            ht_ = np.ctypeslib.as_array(p.hull_tris, (p.hull_nt * 3,)).reshape(p.hull_nt, 3).copy() if p.hull_nt else np.zeros((0, 3), np.int32)
            out.append((v, t, hv_, ht_))
    finally:
        if free:
            _fn("gpu_result_free")(ctypes.byref(res))
    return out


def cand_to_dict(r):
    return {
        "ok": r.ok, "nv": tuple(r.nv), "nt": tuple(r.nt), "n_cap": r.n_cap,
        "hull_nv": tuple(r.hull_nv), "hull_nt": tuple(r.hull_nt),
        "mesh_vol": tuple(r.mesh_vol), "hull_vol": tuple(r.hull_vol),
        "hausdorff": tuple(r.hausdorff), "cost_rv": tuple(r.cost_rv),
        "cost_full": tuple(r.cost_full), "score_rv": r.score_rv,
        "score_full": r.score_full, "err": r.err,
    }
