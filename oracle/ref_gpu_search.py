"""Whole lookahead searches by the reference's own GPU path beside this
library's, on one B200, same meshes and settings.

The reference (eliphatfs/cuacd built from its sources into oracle/_ref by
Makefile.ref) runs through its CPython extension exactly as its Python
wrapper drives it (cuacd/__init__.py:367-454: scipy hull of the input with
outward winding, then `_gpu.lookahead_decompose`).  Two samples, with the
search settings of the benchmark's search legs:

  search   six ridged displaced spheres, tau 0.05, width 30/5, depth 2,
           32 concave edges;
  config4  the 64 meshes with index 0 or 5 mod 16 of config 4's 512 uneven
           meshes, the same with 16 concave edges.

Every mode gets one untimed pass over the search sample first.  Per mesh:
triangles, parts, seconds and the largest part rv cost, for the reference,
this library's exact search and its pruned search (learned level-0 top-48 +
exact beam 8).  Measurement infrastructure only; writes one JSON file.

usage:  python oracle/ref_gpu_search.py out.json [--full]
        (--full: all 512 meshes of config 4 instead of the 64-mesh sample)
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import bench as B  # noqa: E402
import make_ref_gpu as MR  # noqa: E402
from cuacd_b200 import workloads as W  # noqa: E402

KW = dict(max_iters=100, width=30, width2=5, threshold=0.05, depth=2, quick_depth=0, max_n_cutting=16)


def samples(full=False):
    if full:                                          # all 512 meshes of config 4
        return {"search": (B.search_meshes(), 32), "config4_full": (W.batch_meshes(512, 500, 200_000, seed=3), 16)}
    c4 = W.batch_meshes(512, 500, 200_000, seed=3, select={i for i in range(512) if i % 16 in (0, 5)})
    return {"search": (B.search_meshes(), 32), "config4": (c4, 16)}


def ref_search(g, v, t, n_edges):
    import scipy.spatial
    v = np.ascontiguousarray(v, np.float32)
    t = np.ascontiguousarray(t, np.int32)
    t0 = time.perf_counter()
    h = scipy.spatial.ConvexHull(v)
    hv = np.ascontiguousarray(h.points, np.float32)
    ht = np.ascontiguousarray(h.simplices, np.int32)
    cen = hv.mean(0)
    nrm = np.cross(hv[ht[:, 1]] - hv[ht[:, 0]], hv[ht[:, 2]] - hv[ht[:, 0]])
    inward = (nrm * (hv[ht[:, 0]] - cen)).sum(1) < 0
    ht[inward] = ht[inward][:, [0, 2, 1]]
    raw = g.lookahead_decompose(v.ctypes.data, len(v), t.ctypes.data, len(t), hv.ctypes.data, len(hv),
                                ht.ctypes.data, len(ht), KW["max_iters"], KW["width"], KW["width2"],
                                KW["threshold"], KW["depth"], KW["quick_depth"], KW["max_n_cutting"], 0, 0,
                                n_concave_edges=n_edges)
    dt = time.perf_counter() - t0
    parts = []
    for vb, tb, nv, nt, hvb, htb, hnv, hnt, _, _ in raw:
        parts.append((np.frombuffer(vb, np.float32).reshape(nv, 3), np.frombuffer(tb, np.int32).reshape(nt, 3),
                      np.frombuffer(hvb, np.float32).reshape(hnv, 3), np.frombuffer(htb, np.int32).reshape(hnt, 3)))
    return parts, dt


def main(out_path, full=False):
    S = samples(full)
    rec = {"settings": {**KW, "n_concave_edges": {k: e for k, (_, e) in S.items()}}}
    g = MR.load_ref()
    for v, t in S["search"][0]:                       # untimed pass
        ref_search(g, v, t, 32)
    for name, (meshes, ne) in S.items():
        rows = []
        for v, t in meshes:
            try:
                parts, dt = ref_search(g, v, t, ne)
            except Exception as e:                    # record a failed search and go on
                rows.append({"tris": int(len(t)), "parts": 0, "s": 0.0, "max_rv": 0.0, "error": str(e)[:200]})
                continue
            rows.append({"tris": int(len(t)), "parts": len(parts), "s": dt, "max_rv": B.part_cost_max(parts)})
        rec[f"reference_{name}"] = rows
        print("reference", name, sum(r["s"] for r in rows), "s", sum(r["parts"] for r in rows), "parts", flush=True)
    g.destroy()

    import cuacd_b200
    from cuacd_b200 import scorer as SC
    with cuacd_b200.Context(0) as ctx, SC.Scorer.load(ctx, SC.RV_WEIGHTS_PATH) as rv:
        modes = {"exact": {}, "pruned": {"scorer": rv, "top_k": B.SEARCH_TOP_K, "beam": B.SEARCH_BEAM}}
        for mname, extra in modes.items():
            for v, t in S["search"][0]:               # untimed pass
                ctx.lookahead_decompose(v, t, **KW, n_concave_edges=32, **extra)
            for name, (meshes, ne) in S.items():
                rows = []
                for v, t in meshes:
                    t0 = time.perf_counter()
                    try:
                        parts = ctx.lookahead_decompose(v, t, **KW, n_concave_edges=ne, **extra)
                    except RuntimeError as e:
                        rows.append({"tris": int(len(t)), "parts": 0, "s": 0.0, "max_rv": 0.0, "error": str(e)[:200]})
                        continue
                    dt = time.perf_counter() - t0
                    rows.append({"tris": int(len(t)), "parts": len(parts), "s": dt, "max_rv": B.part_cost_max(parts)})
                rec[f"{mname}_{name}"] = rows
                print(mname, name, sum(r["s"] for r in rows), "s", sum(r["parts"] for r in rows), "parts", flush=True)
    with open(out_path, "w") as f:
        json.dump(rec, f)


if __name__ == "__main__":
    main(sys.argv[1], full="--full" in sys.argv[2:])
