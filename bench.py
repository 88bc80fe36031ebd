"""Benchmark: exact candidate evaluation (cut + hull + volume + Hausdorff).

Workload (one step): the 40,960-triangle radially displaced sphere normalised
to extent 2, scored on 30 candidate planes — 27 concave-edge planes (16
concave edges, dihedral > 3.49 rad, cuda/la_concave.cu rule) + 3 axis
midpoints — with the exact evaluator: cut with caps, both fragments' volume
and exact hull, sampled Hausdorff fragment<->hull (2000 samples per unit
area), part costs.  Metric: candidates scored per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value    device-resident throughput (mesh and planes already in HBM), CUDA
         events on the evaluator's stream, L2 flushed (256 MiB write)
         before every timed step; max over ranks for N > 1.
e2e      the same metric through the public C-ABI entry point with pinned
         host buffers (H2D of mesh+planes and D2H of the results per step).
roofline dominant kernel's algorithmic bytes / its CUDA-event duration.
--impl reference: the CPU oracle port of the same path on all host cores
         (the reference has no CPU implementation of this path; its CPU
         baselines need sources absent from the reference tree).
N > 1 runs independent replicas (the path does not shard across GPUs).
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "candidates scored/s (exact: cut+hull+Hausdorff), config 3"
UNIT = "candidates/s"
N_EDGE, WIDTH = 27, 3


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    (profiles/roofline_traffic.txt), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.txt")) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and parts[0] == kernel:
                    return int(parts[1])
    except OSError:
        pass
    return None


def workload():
    from cuacd_b200 import workloads as W
    v, t = W.candidate_mesh()
    return v, t


def planes_for(ctx, v, t):
    """Candidate planes: 16 sampled concave edges -> first 27 planes, plus the
    3 axis midpoints (width 3, margin min(tau/4, 0.015) = 0.0125), generated
    by the library's GPU plane kernels."""
    conc, axis, valid = ctx.candidate_planes(v, t, 16, 0.005, 3.49, WIDTH, 0.0125)
    return np.ascontiguousarray(np.concatenate([conc[:N_EDGE], axis[valid]]).astype(np.float32))


def config(n_planes, v, t):
    return {"workload": "config3: 40,960-tri displaced UV sphere (extent 2, seed 2), "
                        "30 planes (27 concave-edge + 3 axis midpoints), exact evaluator",
            "mesh_tris": int(len(t)), "mesh_verts": int(len(v)), "planes_per_step": int(n_planes),
            "hausdorff_samples": "2000 per unit area, min 1000", "l2": "flushed between timed steps (256 MiB write)",
            "parallelism": "replicas"}


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (getattr(self, "out", "") or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx = float(f[2])
            except ValueError:
                continue
            for n, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(v, t, planes, budget_s=20.0):
    """Oracle port on all host cores over a bounded sample of the workload."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    n = min(len(planes), max(cores, 8))
    t0 = time.perf_counter()
    done = 0
    while True:
        O.eval_candidates(v, t, planes[:n], hausdorff=True, threads=cores)
        done += n
        if time.perf_counter() - t0 > budget_s * 0.5 or done >= 4 * len(planes):
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{done} candidates ({n} planes per pass) of the same workload, "
                      f"oracle (FP64/exact C) with {cores} threads"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import oracle as O
    v, t = workload()
    planes = np.ascontiguousarray(np.concatenate(
        [O.concave_planes(v, t, 16, 0.005, 3.49)[:N_EDGE],
         np.stack([O.axis_plane(v, WIDTH, i, 0.0125) for i in range(WIDTH)])]).astype(np.float32))
    cores = os.cpu_count() or 1
    n = min(len(planes), max(cores, 8))
    for _ in range(args.warmup):
        O.eval_candidates(v, t, planes[:n], hausdorff=True, threads=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.eval_candidates(v, t, planes[:n], hausdorff=True, threads=cores)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    val = n * args.steps / total
    line = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(n, v, t), "impl": "reference",
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{n} of the 30 planes per step, oracle with {cores} threads"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist_.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = dist_

    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import torch
    import cuacd_b200
    lib = cuacd_b200._lib
    lib.cuacd_profile_stages.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.cuacd_stage_times.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    dev = local
    torch.cuda.set_device(dev)
    ctx = cuacd_b200.Context(dev)
    v, t = workload()
    planes = planes_for(ctx, v, t)
    n = len(planes)

    # device-resident inputs
    dv = torch.from_numpy(v.reshape(-1)).cuda()
    dt = torch.from_numpy(t.reshape(-1).astype(np.int32)).cuda()
    dp = torch.from_numpy(planes.reshape(-1)).cuda()
    res_bytes = ctypes.sizeof(cuacd_b200.CandResult) * n
    dres = torch.empty(res_bytes, dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream(device=dev)
    fn_dev = cuacd_b200._fn("cuacd_eval_candidates_device")

    def step():
        rc = fn_dev(ctx.handle, ctypes.c_void_p(dv.data_ptr()), len(v), ctypes.c_void_p(dt.data_ptr()), len(t),
                    ctypes.c_void_p(dp.data_ptr()), n, 1, 2000.0, 1000, 0, ctypes.c_void_p(dres.data_ptr()),
                    ctypes.c_void_p(stream.cuda_stream))
        if rc:
            raise RuntimeError(f"cuacd error {rc}: {lib.gpu_last_error(ctx.handle)}")

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        stream.synchronize()
        # correctness guard on the resident path
        host = (cuacd_b200.CandResult * n)()
        hbuf = dres.cpu().numpy()                 # keep the host copy alive for the memmove
        ctypes.memmove(host, hbuf.ctypes.data, res_bytes)
        n_ok = sum(r.ok for r in host)
        if any(r.err for r in host):
            raise RuntimeError("device evaluation reported errors")

        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        launches0 = ctx.launch_count()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with Clocks(dev) as clk:
            for i in range(args.steps):
                flush.zero_()                       # evict L2 (untimed)
                ev[i][0].record(stream)
                step()
                ev[i][1].record(stream)
            stream.synchronize()
        launches = ctx.launch_count() - launches0
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = [a.elapsed_time(b) for a, b in ev]
        tot_ms = sum(ms)
        # per-stage times (one profiled step, same stream, after the timed loop)
        lib.cuacd_profile_stages(ctx.handle, 1)
        stage_ms = []
        for _ in range(3):
            flush.zero_()
            step()
            arr = (ctypes.c_float * 6)()
            lib.cuacd_stage_times(ctx.handle, ctypes.cast(arr, ctypes.c_void_p))
            stage_ms.append(list(arr))
        lib.cuacd_profile_stages(ctx.handle, 0)
        stage_ms = np.median(np.array(stage_ms), axis=0).tolist()

    # e2e through the public host-pointer entry point with pinned buffers
    pv = torch.from_numpy(v.reshape(-1)).pin_memory()
    pt = torch.from_numpy(t.reshape(-1).astype(np.int32)).pin_memory()
    pp = torch.from_numpy(planes.reshape(-1)).pin_memory()
    pres = torch.empty(res_bytes, dtype=torch.uint8).pin_memory()
    fn_host = cuacd_b200._fn("cuacd_eval_candidates")

    def host_step():
        rc = fn_host(ctx.handle, ctypes.c_void_p(pv.data_ptr()), len(v), ctypes.c_void_p(pt.data_ptr()), len(t),
                     ctypes.c_void_p(pp.data_ptr()), n, 1, 2000.0, 1000, 0, ctypes.c_void_p(pres.data_ptr()))
        if rc:
            raise RuntimeError(f"cuacd error {rc}")

    for _ in range(args.warmup):
        host_step()
    e2e_times = []
    for _ in range(args.steps):
        flush.zero_(); torch.cuda.synchronize()
        t0 = time.perf_counter()
        host_step()
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = sum(e2e_times)

    # max over ranks
    if dist:
        tt = torch.tensor([tot_ms, e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        tot_ms, e2e_s = float(tt[0]), float(tt[1])
    world_n = world
    value = world_n * n * args.steps / (tot_ms / 1000.0)
    e2e_val = world_n * n * args.steps / e2e_s

    # roofline of the dominant stage
    names = ["k_cut_planes", "hull_pipeline", "k_hd_prep", "k_hd_plan", "k_hd_query", "k_eval_finish"]
    dom = int(np.argmax(stage_ms))
    V, T = len(v), len(t)
    Vf = sum(r.nv[0] + r.nv[1] for r in host); Tf = sum(r.nt[0] + r.nt[1] for r in host)
    Hv = sum(r.hull_nv[0] + r.hull_nv[1] for r in host); Ht = sum(r.hull_nt[0] + r.hull_nt[1] for r in host)
    alg = {
        "k_cut_planes": 12 * (V + T) * n + 12 * (Vf + Tf),
        "hull_pipeline": 12 * (Vf + Tf) + 12 * (Hv + Ht),
        "k_hd_prep": 12 * (Vf + Tf) + 12 * (Hv + Ht),
        "k_hd_plan": 0,
        "k_hd_query": 12 * (Vf + Tf) + 12 * (Hv + Ht),
        "k_eval_finish": 0,
    }
    peak, peak_kind = peaks()
    achieved = alg[names[dom]] / (stage_ms[dom] / 1000.0) / 1e9
    roof = {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": ncu_traffic(names[dom]),
            "algorithmic_bytes": int(alg[names[dom]]),
            "stage_ms": {k: round(x, 4) for k, x in zip(names, stage_ms)}}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_n, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (exact int/f64 predicates)",
            "data": "synthetic", "config": config(n, v, t),
            "candidates_ok": int(n_ok), "gpu_launches": int(launches), "clocks": clk.summary(),
            "roofline": roof,
            "e2e": {"value": e2e_val, "unit": UNIT,
                    "h2d_bytes_per_step": int(v.nbytes + t.astype(np.int32).nbytes + planes.nbytes),
                    "d2h_bytes_per_step": int(res_bytes)}}
    if rank == 0 and world_n == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(v, t, planes)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
