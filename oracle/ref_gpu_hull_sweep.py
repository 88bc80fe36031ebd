"""Batched hull volumes: the reference's own GPU path beside this library's,
on one B200, over the batch shapes of the reference's arena sweep
(docs/arena_sweep.md: 10000x20, 1000x200, 100x2000 and 10x20000 points;
sphere shell, cube interior and gaussian clouds; seeded synthetic inputs).

Reference: eliphatfs/cuacd built from its sources into oracle/_ref by
Makefile.ref, driven as its `Context.batch_hull_volume` drives it
(cuacd/__init__.py:185-233): pack, `_gpu.hull_dandc` with output caps of
n / 2n-4 per cloud, then the FP32 volume of every hull on the host.  Both
the `_gpu.hull_dandc` call alone and the whole method are timed.
This library: `Context.batch_hull_volume` (host arrays in and out).
Wall clock per call after one warm-up call, median of five.  The input
index sets of both hulls are compared cloud by cloud.  Measurement
infrastructure only; writes one JSON file.

usage:  python oracle/ref_gpu_hull_sweep.py out.json
"""
import json
import os
import statistics
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import make_ref_gpu as MR  # noqa: E402

SHAPES = [(10000, 20), (1000, 200), (100, 2000), (10, 20000)]
DISTS = ["sphere_shell", "cube_interior", "gaussian"]
REPS = 5


def clouds(n, k, dist, seed):
    rng = np.random.default_rng(seed)
    if dist == "gaussian":
        p = rng.normal(0, 0.5, (n, k, 3))
    elif dist == "cube_interior":
        p = rng.uniform(-1, 1, (n, k, 3))
    else:
        d = rng.normal(size=(n, k, 3))
        p = d / np.linalg.norm(d, axis=2, keepdims=True) * rng.uniform(0.95, 1.0, (n, k, 1))
    p = p.astype(np.float32)
    return [p[i] for i in range(n)]


def ref_batch_hull_volume(g, cl):
    """The reference wrapper's steps; returns (volumes, errors, seconds of
    the _gpu call alone, per-cloud output meshes)."""
    n = len(cl)
    packed = np.ascontiguousarray(np.concatenate(cl), np.float32)
    off = np.zeros(n + 1, np.int32)
    off[1:] = np.cumsum([len(c) for c in cl])
    mhv = max(len(c) for c in cl)
    mht = max(max(2 * len(c) - 4 for c in cl), 4)
    ov = np.empty(n * mhv * 3, np.float32)
    ot = np.empty(n * mht * 3, np.int32)
    onv, ont, err = (np.empty(n, np.int32) for _ in range(3))
    t0 = time.perf_counter()
    g.hull_dandc(packed.ctypes.data, len(packed), off.ctypes.data, n, mhv, mhv, mht, ov.ctypes.data,
                 ot.ctypes.data, onv.ctypes.data, ont.ctypes.data, err.ctypes.data)
    t_call = time.perf_counter() - t0
    vols = np.empty(n, np.float32)
    meshes = []
    for i in range(n):
        hv = ov[i * mhv * 3:(i * mhv + onv[i]) * 3].reshape(-1, 3)
        ht = ot[i * mht * 3:(i * mht + ont[i]) * 3].reshape(-1, 3)
        if len(ht):
            a, b, c = hv[ht[:, 0]], hv[ht[:, 1]], hv[ht[:, 2]]
            vols[i] = abs(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0)
        else:
            vols[i] = 0.0
        meshes.append(hv)
    return vols, err.copy(), t_call, meshes


def main(out_path):
    cases = [(n, k, d, 100 + 10 * si + di) for si, (n, k) in enumerate(SHAPES) for di, d in enumerate(DISTS)]
    data = {c: clouds(*c) for c in cases}
    rows = {c: {"clouds": c[0], "points": c[1], "dist": c[2]} for c in cases}
    g = MR.load_ref()
    for c in cases:
        cl = data[c]
        ref_batch_hull_volume(g, cl)                       # warm-up
        calls, whole = [], []
        for _ in range(REPS):
            t0 = time.perf_counter()
            vols, err, t_call, meshes = ref_batch_hull_volume(g, cl)
            whole.append(time.perf_counter() - t0)
            calls.append(t_call)
        rows[c]["ref_call_ms"] = 1e3 * statistics.median(calls)
        rows[c]["ref_method_ms"] = 1e3 * statistics.median(whole)
        rows[c]["ref_errors"] = int((err != 0).sum())
        rows[c]["_ref_sets"] = [set(MR.index_set(x, m).tolist()) for x, m in zip(cl, meshes)]
        rows[c]["_ref_vol"] = vols
        print("reference", c[:3], round(rows[c]["ref_call_ms"], 2), "ms", flush=True)
    g.destroy()

    import cuacd_b200
    with cuacd_b200.Context(0) as ctx:
        for c in cases:
            cl = data[c]
            ctx.batch_hull_volume(cl)                      # warm-up
            ts = []
            for _ in range(REPS):
                t0 = time.perf_counter()
                vols, err = ctx.batch_hull_volume(cl)
                ts.append(time.perf_counter() - t0)
            rows[c]["ours_ms"] = 1e3 * statistics.median(ts)
            rows[c]["ours_errors"] = int((err != 0).sum())
            meshes = ctx.batch_hull_dandc_mesh(cl)
            ours = [set(MR.index_set(x, m[0]).tolist()) for x, m in zip(cl, meshes)]
            rows[c]["sets_differing"] = int(sum(a != b for a, b in zip(ours, rows[c].pop("_ref_sets"))))
            rv = rows[c].pop("_ref_vol")
            rows[c]["max_rel_vol_diff"] = float(np.max(np.abs(vols - rv) / np.maximum(np.abs(rv), 1e-30)))
            rows[c]["speedup_vs_ref_method"] = rows[c]["ref_method_ms"] / rows[c]["ours_ms"]
            print("ours", c[:3], round(rows[c]["ours_ms"], 2), "ms", "sets differing", rows[c]["sets_differing"],
                  flush=True)
    with open(out_path, "w") as f:
        json.dump(list(rows.values()), f)


if __name__ == "__main__":
    main(sys.argv[1])
