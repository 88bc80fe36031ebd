"""Device allocation throughput: the reference's heap benchmark beside this
library's arena, on one B200.

Reference: bench/malloc_test_bench.cu built from the reference sources by
Makefile.ref into oracle/_ref/malloc_test_bench, run as published (its own
heap, heap_alloc/heap_free, and CUDA's device malloc/free) except for the
iteration count: 256 alloc-free iterations per block instead of 1,024, so
that this library's arena, which frees by whole-arena reset, holds a run's
allocations (1,024 blocks x 256 x 62 KB mean = 16 GB).
This library: `cuacd_arena_bench`, the same workload (grid blocks, thread
0 of each drawing log-uniform sizes in [4 KiB, 256 KiB] into 16 slots),
allocations only, the arena reset before each run.
Both: CUDA events around the kernel, 2 warm-up and 5 timed runs (mean).
One alloc(-free) counts as one op.  Measurement infrastructure only;
writes one JSON file.

usage:  python oracle/ref_gpu_heap_bench.py out.json
"""
import ctypes
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

GRIDS = [1, 4, 16, 64, 256, 1024]
ITERS, SLOTS, SMIN, SMAX = 256, 16, 4096, 262144


def reference_rows():
    r = subprocess.run([os.path.join(HERE, "_ref", "malloc_test_bench"), "--iters", str(ITERS), "--slots", str(SLOTS),
                        "--size-min", str(SMIN), "--size-max", str(SMAX), "--impl", "both"],
                       capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    lines = [l.split(",") for l in r.stdout.splitlines() if l.strip()]
    hdr = lines[0]
    return [dict(zip(hdr, l)) for l in lines[1:]], r.stderr[-1000:]


def main(out_path):
    ref, ref_log = reference_rows()
    import cuacd_b200
    fn = cuacd_b200._lib.cuacd_arena_bench
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_uint,
                   ctypes.c_ulonglong, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                   ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)]
    ours = []
    with cuacd_b200.Context(0) as ctx:
        for g in GRIDS:
            m, s, f = ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
            rc = fn(ctx.handle, g, ITERS, SLOTS, SMIN, SMAX, 20 << 30, 2, 5, ctypes.byref(m), ctypes.byref(s),
                    ctypes.byref(f))
            if rc:
                raise RuntimeError(f"cuacd error {rc}")
            ours.append({"grid": g, "mean_ms": m.value, "std_ms": s.value, "failed_allocs": f.value,
                         "mops": g * ITERS / (m.value * 1e-3) / 1e6})
            print(ours[-1], flush=True)
    rec = {"iters": ITERS, "slots": SLOTS, "size_min": SMIN, "size_max": SMAX, "reference": ref,
           "reference_log": ref_log, "ours": ours}
    with open(out_path, "w") as f:
        json.dump(rec, f)
    for r in ref:
        print(r, flush=True)


if __name__ == "__main__":
    main(sys.argv[1])
