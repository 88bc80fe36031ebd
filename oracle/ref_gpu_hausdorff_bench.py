"""The reference's Hausdorff benchmark beside this library's batched
Hausdorff, on one B200, same meshes.

Reference: bench/hausdorff_bench.cu built from the reference sources by
Makefile.ref into oracle/_ref/hausdorff_bench (GPU rows only; its CPU leg
needs sources absent from the reference tree).  It times `hausdorff_block`,
one block per pair, for the bunny (mesh 4,891 v / 9,790 t vs hull 320 v /
636 t) and the 49160 mesh (278 v / 552 t vs 96 v / 188 t) at batch 1 and
100: CUDA events around the kernel, meshes resident, 2 warm-up and 5 timed
launches (mean).
This library: `cuacd_hausdorff_batch_device` on the same meshes, extracted
from the benchmark's data header into oracle/_ref/hausdorff_bench_data.npz,
the same batches, the same resolution (2000 samples per unit area, at least
1000), CUDA events around the call on its stream, meshes resident, 2
warm-up and 5 timed calls (mean).  Measurement infrastructure only; writes
one JSON file.

usage:  python oracle/ref_gpu_hausdorff_bench.py out.json
"""
import ctypes
import json
import os
import statistics
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
REF = os.path.join(HERE, "_ref")


def reference_rows():
    r = subprocess.run([os.path.join(REF, "hausdorff_bench")], capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    lines = [l.split(",") for l in r.stdout.splitlines() if l.strip()]
    hdr = lines[0]
    rows = [dict(zip(hdr, l)) for l in lines[1:]]
    return [x for x in rows if x["algorithm"] == "hausdorff_block"]


def ours(ctx, mesh, hull, batch):
    import torch
    import cuacd_b200
    fn = cuacd_b200._fn("cuacd_hausdorff_batch_device")
    (mv, mt), (hv, ht) = mesh, hull
    dav = torch.from_numpy(np.ascontiguousarray(np.tile(mv, (batch, 1)), np.float32)).cuda()
    dat = torch.from_numpy(np.ascontiguousarray(np.tile(mt, (batch, 1)), np.int32)).cuda()
    dbv = torch.from_numpy(np.ascontiguousarray(np.tile(hv, (batch, 1)), np.float32)).cuda()
    dbt = torch.from_numpy(np.ascontiguousarray(np.tile(ht, (batch, 1)), np.int32)).cuda()
    avo = np.arange(batch + 1, dtype=np.int32) * len(mv)
    ato = np.arange(batch + 1, dtype=np.int32) * len(mt)
    bvo = np.arange(batch + 1, dtype=np.int32) * len(hv)
    bto = np.arange(batch + 1, dtype=np.int32) * len(ht)
    out = torch.zeros(batch, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    P = ctypes.c_void_p

    def call():
        rc = fn(ctx.handle, batch, P(dav.data_ptr()), P(avo.ctypes.data), P(dat.data_ptr()), P(ato.ctypes.data),
                P(dbv.data_ptr()), P(bvo.ctypes.data), P(dbt.data_ptr()), P(bto.ctypes.data), 2000.0, 1000, 0,
                P(out.data_ptr()), P(stream.cuda_stream))
        if rc:
            raise RuntimeError(f"cuacd error {rc}")

    for _ in range(2):
        call()
    ms = []
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        call()
        b.record(stream)
        stream.synchronize()
        ms.append(a.elapsed_time(b))
    d = out.cpu().numpy()
    return statistics.mean(ms), statistics.pstdev(ms), float(d.mean()), float(d.max() - d.min())


def main(out_path):
    ref = reference_rows()
    import cuacd_b200
    data = np.load(os.path.join(REF, "hausdorff_bench_data.npz"))
    sets = {"bunny": "BUNNY", "49160": "STL"}
    rows = []
    with cuacd_b200.Context(0) as ctx:
        for r in ref:
            k = sets[r["dataset"]]
            batch = int(r["batch"])
            m, s, dist, spread = ours(ctx, (data[f"{k}_verts"], data[f"{k}_tris"]),
                                      (data[f"{k}_hull_verts"], data[f"{k}_hull_tris"]), batch)
            rows.append({"dataset": r["dataset"], "batch": batch, "ref_ms": float(r["mean_ms"]),
                         "ref_std_ms": float(r["std_ms"]), "ref_dist": float(r["mean_dist"]), "ours_ms": m,
                         "ours_std_ms": s, "ours_dist": dist, "ours_dist_spread": spread,
                         "speedup": float(r["mean_ms"]) / m})
            print(rows[-1], flush=True)
    with open(out_path, "w") as f:
        json.dump(rows, f)


if __name__ == "__main__":
    main(sys.argv[1])
