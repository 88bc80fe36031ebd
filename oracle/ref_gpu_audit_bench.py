"""Mesh audit: the reference's own GPU audit beside this library's, one
B200, same meshes.  Reference: `_gpu.mesh_audit` of eliphatfs/cuacd built
from its sources by Makefile.ref (one 256-thread block per mesh).  This
library: `Context.check_mesh` (gpu_mesh_audit).  Wall clock of the public
call, host arrays in, verdict out; median of 5 after one warm-up.
Measurement infrastructure only; writes one JSON file.

usage:  python oracle/ref_gpu_audit_bench.py out.json
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
from cuacd_b200 import workloads as W  # noqa: E402


def meshes():
    big = [m for m in W.batch_meshes(512, 500, 200_000, seed=3, select={i for i in range(512) if i % 16 in (0, 5)})
           if len(m[1]) == 327680][0]
    return [("40,960-tri sphere", *W.candidate_mesh()), ("327,680-tri sphere", *big)]


def timed(fn):
    fn()
    ts = []
    for _ in range(5):
        t0 = time.perf_counter()
        r = fn()
        ts.append(time.perf_counter() - t0)
    return 1e3 * statistics.median(ts), r


def main(out_path):
    ms = [(n, np.ascontiguousarray(v, np.float32), np.ascontiguousarray(t, np.int32)) for n, v, t in meshes()]
    rows = []
    g = MR.load_ref()
    for n, v, t in ms:
        ref_ms, ref_f = timed(lambda: g.mesh_audit(v.ctypes.data, len(v), t.ctypes.data, len(t)))
        rows.append({"mesh": n, "tris": int(len(t)), "ref_ms": ref_ms, "ref_flags": int(ref_f)})
    g.destroy()
    import cuacd_b200
    with cuacd_b200.Context(0) as ctx:
        for row, (n, v, t) in zip(rows, ms):
            ours_ms, r = timed(lambda: ctx.check_mesh(v, t))
            row.update({"ours_ms": ours_ms, "ours_flags": r["flags"], "speedup": row["ref_ms"] / ours_ms})
            print(row, flush=True)
    with open(out_path, "w") as f:
        json.dump(rows, f)


if __name__ == "__main__":
    main(sys.argv[1])
