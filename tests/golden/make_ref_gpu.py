"""Record the reference's own GPU outputs as golden fixtures.

Runs eliphatfs/cuacd's CUDA path -- its kernels.fatbin and CPython host
extension, built from the reference sources by `oracle/Makefile.ref` into
oracle/_ref/ -- on a B200, through the extension's own entry points
(`_gpu.hull_dandc`, `kdop_hull`, `batch_mesh_volume`, `test_plane_cut`,
`test_hausdorff`, `lookahead_decompose`; csrc/module.c in the reference), on
the seeded inputs of `cases()` below, and writes what they return to one
small .npz.  The fixture is committed (tests/golden/ref_gpu.npz); the tests
regenerate the inputs from the same seeds and compare the oracle (CPU) and
this library's CUDA path (GPU) with the reference's results.

usage (on a machine with a B200, after `make -f oracle/Makefile.ref REF=...`):
    python tests/golden/make_ref_gpu.py [out.npz]
    python tests/golden/make_ref_gpu.py --audit [out.npz]    (mesh-audit verdicts: ref_gpu_audit.npz)
    python tests/golden/make_ref_gpu.py --concave [out.npz]  (concave-edge planes: ref_gpu_concave.npz)
    python tests/golden/make_ref_gpu.py --search [out.npz]   (config-4 sample searches: ref_gpu_search.npz)
"""
import importlib.machinery
import importlib.util
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..", "..")
sys.path.insert(0, ROOT)


def _workloads():
    """cuacd_b200/workloads.py (plain numpy) loaded by path, so that this
    process, which runs the reference, never maps this library."""
    spec = importlib.util.spec_from_file_location("_cuacd_workloads", os.path.join(ROOT, "cuacd_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


W = _workloads()

REF_DIR = os.path.join(ROOT, "oracle", "_ref")


# ---------------------------------------------------------------------------
# inputs (shared with the tests)
# ---------------------------------------------------------------------------

def hull_cases():
    """(name, list of float32 clouds) for hull_dandc."""
    rng = np.random.default_rng(10)
    gauss = [rng.normal(0, 0.5, (2000, 3)).astype(np.float32) for _ in range(16)]
    rng = np.random.default_rng(11)
    shell = []
    for _ in range(8):
        d = rng.normal(size=(3000, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        shell.append((d * rng.uniform(0.9, 1.0, (3000, 1))).astype(np.float32))
    big = W.hull_clouds(4, 20000, 12)
    return [("uniform_1000", W.hull_clouds(256, 1000, 0)), ("gauss_2000", gauss),
            ("shell_3000", shell), ("uniform_20000", big)]


def kdop_clouds():
    v3, _ = W.candidate_mesh(64, 24)
    vh, _ = W.hausdorff_sphere(level=4)
    return W.hull_clouds(4, 20000, 12) + [v3, vh]


def volume_meshes():
    iv, it = W.icosphere(3)
    return [(iv.astype(np.float32), it.astype(np.int32)), W.hausdorff_sphere(level=4), W.candidate_mesh(),
            W.candidate_mesh(64, 24), W.box((-1, -0.5, -0.25), (1, 0.5, 0.25), 3)]


def cut_cases():
    """(mesh, planes): the 40,960-triangle sphere and a small one, each with
    the three axis midplanes and eight seeded oblique planes."""
    out = []
    for k, (v, t) in enumerate([W.candidate_mesh(), W.candidate_mesh(64, 24)]):
        rng = np.random.default_rng(20 + k)
        planes = [[1, 0, 0, -0.011], [0, 1, 0, 0.013], [0, 0, 1, -0.007]]
        for _ in range(8):
            n = rng.normal(size=3)
            n /= np.linalg.norm(n)
            planes.append([*n, rng.uniform(-0.4, 0.4)])
        out.append((v, t.astype(np.int32), np.array(planes, np.float32)))
    return out


def hausdorff_meshes():
    """Meshes whose (reference hull, mesh) pairs go through test_hausdorff."""
    iv, it = W.icosphere(3)
    return [W.hausdorff_sphere(level=3), W.candidate_mesh(64, 24), (iv.astype(np.float32), it.astype(np.int32))]


def lookahead_meshes():
    return [W.candidate_mesh(64, 24), W.candidate_mesh(96, 32, 0.35, seed=5)]


def audit_cases():
    """(name, verts, tris) for the topology audit: closed meshes and the
    same meshes broken in each way the verdict bits name."""
    v, t = W.candidate_mesh(64, 24)
    t = t.astype(np.int32)
    bv, bt = W.box((-1, -0.5, -0.25), (1, 0.5, 0.25), 3)
    rng = np.random.default_rng(30)
    mv, mt = W.random_boxes_mesh(4, 3000, rng)
    big = [m for m in W.batch_meshes(512, 500, 200_000, seed=3, select={i for i in range(512) if i % 16 in (0, 5)})
           if len(m[1]) == 327680][0]
    flip = t.copy(); flip[100] = flip[100][[0, 2, 1]]
    extra_v = np.concatenate([v, np.array([[3.0, 3.0, 3.0]], np.float32)])
    nonman = np.concatenate([t, np.array([[t[0, 0], t[0, 1], len(v)]], np.int32)])
    col_v = np.concatenate([v, np.array([[0, 0, 0], [1, 1, 1], [2, 2, 2]], np.float32)])
    collinear = np.concatenate([t, np.array([[len(v), len(v) + 1, len(v) + 2]], np.int32)])
    rep = np.concatenate([t, np.array([[5, 5, 6]], np.int32)])
    bad = np.concatenate([t, np.array([[0, 1, len(v)]], np.int32)])
    neg = np.concatenate([t, np.array([[0, -1, 2]], np.int32)])
    dup = np.concatenate([t, t[:1]])
    bflip = big[1].astype(np.int32).copy(); bflip[5000] = bflip[5000][[1, 0, 2]]
    return [("sphere", v, t), ("box", bv, bt.astype(np.int32)), ("boxes", mv, mt.astype(np.int32)),
            ("open", v, t[:-1]), ("flipped", v, flip), ("nonmanifold", extra_v, nonman),
            ("collinear", col_v, collinear), ("repeated_index", v, rep), ("bad_index", v, bad),
            ("negative_index", v, neg), ("duplicate_triangle", v, dup), ("big_sphere", big[0], big[1].astype(np.int32)),
            ("big_flipped", big[0], bflip)]


def main_audit(out_path):
    """The reference's `_gpu.mesh_audit` verdict on every audit case."""
    g = load_ref()
    rec = {}
    for name, v, t in audit_cases():
        v = np.ascontiguousarray(v, np.float32)
        t = np.ascontiguousarray(t, np.int32)
        rec[name] = np.array([g.mesh_audit(v.ctypes.data, len(v), t.ctypes.data, len(t))], np.uint32)
        print(name, int(rec[name][0]), flush=True)
    g.destroy()
    np.savez_compressed(out_path, **rec)


LOOKAHEAD_KW = dict(max_iters=100, width=30, width2=5, threshold=0.05, depth=2, quick_depth=0,
                    max_n_cutting=16, n_concave_edges=16)


# ---------------------------------------------------------------------------
# reference driver
# ---------------------------------------------------------------------------

def load_ref():
    path = os.path.join(REF_DIR, "_gpu.so")
    loader = importlib.machinery.ExtensionFileLoader("_gpu", path)
    spec = importlib.util.spec_from_loader("_gpu", loader)
    g = importlib.util.module_from_spec(spec)
    loader.exec_module(g)
    with open(os.path.join(REF_DIR, "kernels.fatbin"), "rb") as f:
        g.set_fatbin(f.read())
    g.init(0, 8 << 30)
    return g


def index_set(cloud, hv):
    """Input indices of the hull's vertices (the reference copies input
    floats into its output, so each output vertex names an input point)."""
    key = {tuple(p): i for i, p in reversed(list(enumerate(map(tuple, cloud))))}
    return np.array(sorted(key[tuple(p)] for p in map(tuple, hv)), np.int32)


def vol64(v, t):
    v = np.asarray(v, np.float64)
    a, b, c = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    return float(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0)


def ref_hull(g, clouds, kdop=False):
    n = len(clouds)
    packed = np.ascontiguousarray(np.concatenate(clouds).astype(np.float32))
    off = np.zeros(n + 1, np.int32)
    off[1:] = np.cumsum([len(c) for c in clouds])
    if kdop:
        mhv, mht = 4096, 8192
    else:
        mhv, mht = max(len(c) for c in clouds), max(max(2 * len(c) - 4 for c in clouds), 4)
    ov = np.empty(n * mhv * 3, np.float32)
    ot = np.empty(n * mht * 3, np.int32)
    onv, ont, err = (np.empty(n, np.int32) for _ in range(3))
    ovol = np.empty(n, np.float32)
    if kdop:
        g.kdop_hull(packed.ctypes.data, len(packed), off.ctypes.data, n, mhv, mht, ov.ctypes.data, ot.ctypes.data,
                    onv.ctypes.data, ont.ctypes.data, ovol.ctypes.data, err.ctypes.data)
    else:
        g.hull_dandc(packed.ctypes.data, len(packed), off.ctypes.data, n, max(len(c) for c in clouds), mhv, mht,
                     ov.ctypes.data, ot.ctypes.data, onv.ctypes.data, ont.ctypes.data, err.ctypes.data)
    res = []
    for i, c in enumerate(clouds):
        hv = ov[i * mhv * 3:(i * mhv + onv[i]) * 3].reshape(-1, 3)
        ht = ot[i * mht * 3:(i * mht + ont[i]) * 3].reshape(-1, 3)
        res.append((index_set(c, hv), int(onv[i]), int(ont[i]), int(err[i]), vol64(hv, ht) if len(ht) else 0.0,
                    float(ovol[i]) if kdop else np.nan, hv.copy(), ht.copy()))
    return res


def ref_cut(g, v, t, p):
    nv, nt = len(v), len(t)
    vcap, tcap = nv + 2 * nt, 3 * nt + 64
    pv, nvv = np.empty(vcap * 3, np.float32), np.empty(vcap * 3, np.float32)
    pt, ntt = np.empty(tcap * 3, np.int32), np.empty(tcap * 3, np.int32)
    v = np.ascontiguousarray(v, np.float32)
    t = np.ascontiguousarray(t, np.int32)
    a, b, c, d = (float(x) for x in p)
    n_pv, n_pt, n_nv, n_nt = g.test_plane_cut(v.ctypes.data, nv, t.ctypes.data, nt, a, b, c, d,
                                              pv.ctypes.data, vcap, pt.ctypes.data, tcap,
                                              nvv.ctypes.data, vcap, ntt.ctypes.data, tcap)
    vp = vol64(pv[:3 * n_pv].reshape(-1, 3), pt[:3 * n_pt].reshape(-1, 3)) if n_pt else 0.0
    vn = vol64(nvv[:3 * n_nv].reshape(-1, 3), ntt[:3 * n_nt].reshape(-1, 3)) if n_nt else 0.0
    return [n_pv, n_pt, n_nv, n_nt], [vp, vn]


def ref_hausdorff(g, a, b):
    av, at = (np.ascontiguousarray(x) for x in (a[0].astype(np.float32), a[1].astype(np.int32)))
    bv, bt = (np.ascontiguousarray(x) for x in (b[0].astype(np.float32), b[1].astype(np.int32)))
    out = np.zeros(1, np.float32)
    g.test_hausdorff(av.ctypes.data, len(av), at.ctypes.data, len(at), bv.ctypes.data, len(bv),
                     bt.ctypes.data, len(bt), out.ctypes.data)
    return float(out[0])


def ref_lookahead(g, v, t):
    import scipy.spatial
    v = np.ascontiguousarray(v, np.float32)
    t = np.ascontiguousarray(t, np.int32)
    h = scipy.spatial.ConvexHull(v)
    hv = np.ascontiguousarray(h.points, np.float32)
    ht = np.ascontiguousarray(h.simplices, np.int32)
    # outward winding, as the reference's Python wrapper arranges it
    cen = hv.mean(0)
    nrm = np.cross(hv[ht[:, 1]] - hv[ht[:, 0]], hv[ht[:, 2]] - hv[ht[:, 0]])
    inward = (nrm * (hv[ht[:, 0]] - cen)).sum(1) < 0
    ht[inward] = ht[inward][:, [0, 2, 1]]
    kw = LOOKAHEAD_KW
    t0 = time.perf_counter()
    raw = g.lookahead_decompose(v.ctypes.data, len(v), t.ctypes.data, len(t), hv.ctypes.data, len(hv),
                                ht.ctypes.data, len(ht), kw["max_iters"], kw["width"], kw["width2"],
                                kw["threshold"], kw["depth"], kw["quick_depth"], kw["max_n_cutting"], 0, 0,
                                n_concave_edges=kw["n_concave_edges"])
    dt = time.perf_counter() - t0
    return [(float(r[8]), float(r[9])) for r in raw], dt


def main(out_path):
    g = load_ref()
    rec = {}
    for name, clouds in hull_cases():
        res = ref_hull(g, clouds)
        rec[f"hull_{name}_idx"] = np.concatenate([r[0] for r in res])
        rec[f"hull_{name}_off"] = np.cumsum([0] + [len(r[0]) for r in res]).astype(np.int32)
        rec[f"hull_{name}_nvnterr"] = np.array([[r[1], r[2], r[3]] for r in res], np.int32)
        rec[f"hull_{name}_vol"] = np.array([r[4] for r in res])
        print(name, "errors", int(sum(r[3] != 0 for r in res)), flush=True)
    res = ref_hull(g, kdop_clouds(), kdop=True)
    rec["kdop_idx"] = np.concatenate([r[0] for r in res])
    rec["kdop_off"] = np.cumsum([0] + [len(r[0]) for r in res]).astype(np.int32)
    rec["kdop_nvnterr"] = np.array([[r[1], r[2], r[3]] for r in res], np.int32)
    rec["kdop_vol"] = np.array([r[5] for r in res])
    meshes = volume_meshes()
    vv = [np.ascontiguousarray(m[0], np.float32) for m in meshes]
    tt = [np.ascontiguousarray(m[1], np.int32) for m in meshes]
    allv, allt = np.concatenate(vv), np.concatenate(tt)
    voff = np.cumsum([0] + [len(x) for x in vv]).astype(np.int32)
    toff = np.cumsum([0] + [len(x) for x in tt]).astype(np.int32)
    vols = np.empty(len(meshes), np.float32)
    g.batch_mesh_volume(allv.ctypes.data, len(allv), allt.ctypes.data, len(allt), toff.ctypes.data,
                        voff.ctypes.data, len(meshes), vols.ctypes.data)
    rec["mesh_volume"] = vols
    for k, (v, t, planes) in enumerate(cut_cases()):
        cnt, vol = zip(*[ref_cut(g, v, t, p) for p in planes])
        rec[f"cut{k}_counts"] = np.array(cnt, np.int32)
        rec[f"cut{k}_vols"] = np.array(vol)
    for k, (v, t) in enumerate(hausdorff_meshes()):
        (_, _, _, _, _, _, hv, ht), = ref_hull(g, [v])
        rec[f"hd{k}_hull_v"], rec[f"hd{k}_hull_t"] = hv, ht
        rec[f"hd{k}_dist"] = np.array([ref_hausdorff(g, (hv, ht), (v, t))])
    np.savez_compressed(out_path, **rec)          # the lookahead runs below are the longest
    for k, (v, t) in enumerate(lookahead_meshes()):
        parts, dt = ref_lookahead(g, v, t)
        rec[f"la{k}_parts"] = np.array(parts, np.float64).reshape(-1, 2)
        rec[f"la{k}_seconds"] = np.array([dt])
        print("lookahead", k, len(parts), "parts", round(dt, 3), "s", flush=True)
    g.destroy()
    np.savez_compressed(out_path, **rec)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


CONCAVE_KW = dict(eps=0.005, threshold=3.49)


def concave_cases():
    """(name, verts, tris, n_concave_edges): the config-3 sphere with its 16
    sampled edges, the six ridged spheres of the search sample with 16 and
    with 32, and the first displaced sphere of the config-4 sample (smooth:
    no edge passes the dihedral test)."""
    import bench as B
    v3, t3 = W.candidate_mesh()
    out = [("config3", v3, t3, 16)]
    for k, (v, t) in enumerate(B.search_meshes()):
        out += [(f"search{k}_16", v, t, 16), (f"search{k}_32", v, t, 32)]
    c4 = W.batch_meshes(512, 500, 200_000, seed=3, select={0})
    out.append(("config4_0", c4[0][0], c4[0][1], 16))
    return [(n, np.ascontiguousarray(v, np.float32), np.ascontiguousarray(t, np.int32), e) for n, v, t, e in out]


def main_concave(out_path):
    """The planes the reference's la_find_concave_edges emits for each case,
    through oracle/_ref/ref_concave.so (its kernel launched on a one-part
    decomposition state, its own context set-up)."""
    import ctypes
    lib = ctypes.CDLL(os.path.join(REF_DIR, "ref_concave.so"))
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    lib.gpu_set_fatbin.argtypes = [P, ctypes.c_size_t]
    lib.gpu_init.argtypes = [ctypes.POINTER(P), I, ctypes.c_size_t]
    lib.ref_concave_planes.argtypes = [P, P, I, P, I, I, F, F, P, ctypes.POINTER(I), ctypes.POINTER(I)]
    with open(os.path.join(REF_DIR, "kernels.fatbin"), "rb") as f:
        fat = f.read()
    fat_buf = ctypes.create_string_buffer(fat, len(fat))
    lib.gpu_set_fatbin(fat_buf, len(fat))
    ctx = P()
    rc = lib.gpu_init(ctypes.byref(ctx), 0, 2 << 30)
    assert rc == 0, rc
    rec = {}
    for name, v, t, ne in concave_cases():
        out = np.zeros((4 * ne, 4), np.float32)
        n, err = I(0), I(0)
        rc = lib.ref_concave_planes(ctx, v.ctypes.data, len(v), t.ctypes.data, len(t), ne, CONCAVE_KW["eps"],
                                    CONCAVE_KW["threshold"], out.ctypes.data, ctypes.byref(n), ctypes.byref(err))
        assert rc == 0 and err.value == 0, (name, rc, err.value)
        rec[f"{name}_planes"] = out[:n.value].copy()
        rec[f"{name}_n_edges"] = np.array([ne], np.int32)
        print(name, n.value, "planes", flush=True)
    np.savez_compressed(out_path, **rec)


def main_search(out_path):
    """Per mesh of config 4's 64-mesh sample: the reference's part count and
    its largest part rv cost (FP64 volumes) under config 4's settings."""
    g = load_ref()
    c4 = W.batch_meshes(512, 500, 200_000, seed=3, select={i for i in range(512) if i % 16 in (0, 5)})
    parts, worst = [], []
    for v, t in c4:
        raw = ref_lookahead_parts(g, v, t)
        parts.append(len(raw))
        w = 0.0
        for pv, pt, hv, ht in raw:
            gap = max(abs(vol64(hv, ht)) - abs(vol64(pv, pt)), 0.0) if len(ht) else 0.0
            w = max(w, 0.3 * np.cbrt(3.0 / (4.0 * np.pi) * gap))
        worst.append(w)
    g.destroy()
    np.savez_compressed(out_path, parts=np.array(parts, np.int32), max_rv=np.array(worst),
                        tris=np.array([len(t) for _, t in c4], np.int32))
    print("parts", sum(parts), "max rv", max(worst), flush=True)


def ref_lookahead_parts(g, v, t):
    """The reference's lookahead_decompose as its wrapper drives it, with
    LOOKAHEAD_KW; the parts as (verts, tris, hull verts, hull tris)."""
    import scipy.spatial
    v = np.ascontiguousarray(v, np.float32)
    t = np.ascontiguousarray(t, np.int32)
    h = scipy.spatial.ConvexHull(v)
    hv = np.ascontiguousarray(h.points, np.float32)
    ht = np.ascontiguousarray(h.simplices, np.int32)
    cen = hv.mean(0)
    nrm = np.cross(hv[ht[:, 1]] - hv[ht[:, 0]], hv[ht[:, 2]] - hv[ht[:, 0]])
    inward = (nrm * (hv[ht[:, 0]] - cen)).sum(1) < 0
    ht[inward] = ht[inward][:, [0, 2, 1]]
    kw = LOOKAHEAD_KW
    raw = g.lookahead_decompose(v.ctypes.data, len(v), t.ctypes.data, len(t), hv.ctypes.data, len(hv),
                                ht.ctypes.data, len(ht), kw["max_iters"], kw["width"], kw["width2"],
                                kw["threshold"], kw["depth"], kw["quick_depth"], kw["max_n_cutting"], 0, 0,
                                n_concave_edges=kw["n_concave_edges"])
    out = []
    for vb, tb, nv, nt, hvb, htb, hnv, hnt, _, _ in raw:
        out.append((np.frombuffer(vb, np.float32).reshape(nv, 3), np.frombuffer(tb, np.int32).reshape(nt, 3),
                    np.frombuffer(hvb, np.float32).reshape(hnv, 3), np.frombuffer(htb, np.int32).reshape(hnt, 3)))
    return out


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--audit":
        main_audit(sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, "ref_gpu_audit.npz"))
    elif len(sys.argv) > 1 and sys.argv[1] == "--concave":
        main_concave(sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, "ref_gpu_concave.npz"))
    elif len(sys.argv) > 1 and sys.argv[1] == "--search":
        main_search(sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, "ref_gpu_search.npz"))
    else:
        main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_gpu.npz"))
