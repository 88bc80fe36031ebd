"""Benchmark: candidate scoring, surrogate-pruned vs exact.

Workload (one step): the 40,960-triangle radially displaced sphere normalised
to extent 2, scored on 30 candidate planes — 27 concave-edge planes (16
concave edges, dihedral > 3.49 rad, cuda/la_concave.cu rule) + 3 axis
midpoints.  The exact evaluator cuts with caps, computes both fragments'
volume and exact hull, the sampled Hausdorff distance fragment<->hull (2000
samples per unit area) and the part costs.  The surrogate-pruned step ranks
all 30 planes with the learned scorer (GPU feature rows + BF16 tensor-core
MLP) and sends the top 8, plus every plane predicted within 0.005 of the
8th, through the exact evaluator.  Metric: candidates scored per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value    surrogate-pruned throughput, device-resident (mesh and planes
         already in HBM), CUDA events on the evaluator's stream, L2 flushed
         (256 MiB write) before every timed step; max over ranks for N > 1.
         "exact" holds the same numbers for the exact evaluator on all 30
         planes; "pruning" the planes evaluated exactly and whether the
         pruned step found the exact step's best plane.
e2e      the same metric through the public C-ABI entry point with pinned
         host buffers (H2D of mesh+planes and D2H of the results per step).
roofline dominant kernel's algorithmic bytes / its CUDA-event duration.
--impl reference: the CPU oracle port of the exact path on all host cores
         (the reference has no CPU implementation of this path; its CPU
         baselines need sources absent from the reference tree).
search   whole lookahead searches on six ridged spheres through the host API:
         meshes/s exact vs pruned (learned level-0 ranking + exact beam),
         part counts and the largest part cost of each.
config4  the same on a 64-mesh sample of config 4's uneven batch.
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

METRIC = "candidates scored/s at tau=0.05 on 1 B200: surrogate-pruned vs exact (config 3)"
UNIT = "candidates/s"
N_EDGE, WIDTH = 27, 3
TOP_K, MARGIN = 8, 0.005


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel, planes):
    """DRAM bytes per launch of `kernel` on a step of `planes` candidate
    planes, from the committed ncu summary (profiles/roofline_traffic.txt:
    lines "kernel planes bytes"), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.txt")) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 3 and parts[0] == kernel and parts[1] == str(planes):
                    return int(parts[2])
    except OSError:
        pass
    return None


def ncu_counters(stage):
    """Issue efficiency, cache hit rates and DRAM throughput of the stage's
    main kernel from the committed ncu summary (profiles/roofline_traffic.txt:
    lines "counters stage kernel l2 l1 issue warps dram"), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.txt")) as f:
            for line in f:
                p = line.split()
                if len(p) == 8 and p[0] == "counters" and p[1] == stage:
                    return {"kernel": p[2], "l2_hit_pct": float(p[3]), "l1_hit_pct": float(p[4]),
                            "issue_active_pct": float(p[5]), "warps_active_pct": float(p[6]),
                            "dram_throughput_pct": float(p[7]), "source": "profiles/eval_config3_kernels_full.md"}
    except (OSError, ValueError):
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
                        "30 planes (27 concave-edge + 3 axis midpoints); learned scorer ranks all 30, "
                        "exact evaluator on the top 8 (+ margin 0.005)",
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


SEARCH_TOP_K, SEARCH_BEAM = 48, 8


def search_meshes():
    """Search sample: six ridged displaced spheres (UV 64x24, 96x32, 128x40
    and icospheres of 5,120-20,480 triangles), extent 2; their creases give
    the concave-edge planes the search ranks."""
    from cuacd_b200 import workloads as W
    out = [W.candidate_mesh(64, 24), W.candidate_mesh(96, 32, 0.35, seed=5), W.candidate_mesh(128, 40, 0.4, seed=7)]
    for lvl, amp, sd in ((4, 0.35, 1), (4, 0.45, 2), (5, 0.4, 3)):
        v, t = W.icosphere(lvl)
        v, t = W.displaced_sphere(v, t, amp, sd, n_terms=6, fmin=2.0, fmax=5.0, ridged=True)
        out.append((W.normalize_extent(v).astype(np.float32), t))
    return out


def part_cost_max(parts):
    """Largest rv cost of the returned parts (FP64 volumes of part and hull)."""
    worst = 0.0
    for v, t, hv, ht in parts:
        def vol(V, T):
            V = V.astype(np.float64)
            return abs(float(np.einsum("ij,ij->i", V[T[:, 0]], np.cross(V[T[:, 1]], V[T[:, 2]])).sum()) / 6.0)
        g = max(vol(hv, ht) - vol(v, t), 0.0) if len(ht) else 0.0
        worst = max(worst, 0.3 * np.cbrt(3.0 / (4.0 * np.pi) * g))
    return worst


def search_leg(ctx, scorer, untrained):
    """Whole lookahead searches (tau 0.05, width 30/5, depth 2, 32 concave
    edges) on the search sample through the host API, exact and pruned (the
    level-0 scorer keeps the top 48 planes of each part, the exact search
    then expands the 8 best level-0 cuts).  One untimed pass of each mode
    over the sample first (pools grow to size).  Ablations: the same beam without the
    scorer, and the same pruning with an untrained (random) network."""
    kw = dict(width=30, width2=5, depth=2, threshold=0.05, max_iters=100)
    modes = {"exact": {}, "pruned": {"scorer": scorer, "top_k": SEARCH_TOP_K, "beam": SEARCH_BEAM},
             "beam_only": {"beam": SEARCH_BEAM},
             "untrained": {"scorer": untrained, "top_k": SEARCH_TOP_K, "beam": SEARCH_BEAM}}
    meshes = search_meshes()
    out = {}
    for name, extra in modes.items():
        for v, t in meshes:                       # untimed: the pools grow to the largest mesh's needs
            ctx.lookahead_decompose(v, t, **kw, **extra)
        t0 = time.perf_counter()
        parts = [ctx.lookahead_decompose(v, t, **kw, **extra) for v, t in meshes]
        dt = time.perf_counter() - t0
        out[name] = {"meshes_per_s": len(meshes) / dt, "s": dt, "parts": int(sum(len(p) for p in parts)),
                     "max_rv_cost": float(max(part_cost_max(p) for p in parts))}
    out["speedup"] = out["exact"]["s"] / out["pruned"]["s"]
    out["parts_ratio"] = out["pruned"]["parts"] / max(out["exact"]["parts"], 1)
    out["workload"] = (f"{len(meshes)} ridged displaced spheres (3,072-20,480 tris), tau 0.05, width 30/5, "
                       f"depth 2, 32 concave edges; pruned = learned top-{SEARCH_TOP_K} + beam {SEARCH_BEAM}")
    return out


def config4_leg(ctx, scorer):
    """Config 4 sample: the 64 meshes with index 0 or 5 mod 16 of the 512
    uneven synthetic meshes (500 to 200,000 triangles; displaced icospheres
    and unions of 2-6 boxes, seed 3), whole searches with config 4's
    parameters (tau 0.05, width 30/5, depth 2, 16 concave edges), exact and
    pruned; one untimed pass first."""
    from cuacd_b200 import workloads as W
    meshes = W.batch_meshes(512, 500, 200_000, seed=3, select={i for i in range(512) if i % 16 in (0, 5)})
    kw = dict(width=30, width2=5, depth=2, threshold=0.05, max_iters=100, n_concave_edges=16)
    out = {}
    for name, extra in (("exact", {}), ("pruned", {"scorer": scorer, "top_k": SEARCH_TOP_K, "beam": SEARCH_BEAM})):
        for v, t in meshes:
            ctx.lookahead_decompose(v, t, **kw, **extra)
        t0 = time.perf_counter()
        parts = [ctx.lookahead_decompose(v, t, **kw, **extra) for v, t in meshes]
        dt = time.perf_counter() - t0
        out[name] = {"meshes_per_s": len(meshes) / dt, "s": dt, "parts": int(sum(len(p) for p in parts)),
                     "max_rv_cost": float(max(part_cost_max(p) for p in parts))}
    out["workload"] = (f"config 4 sample: {len(meshes)} of the 512 meshes (index 0 or 5 mod 16), "
                       f"{min(len(t) for _, t in meshes)}-{max(len(t) for _, t in meshes)} tris")
    return out


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


def replica_max(totals, dist, device):
    """Per-rank totals (times) -> their maximum over the ranks: N replicas
    finish when the slowest one does.  Without a process group, unchanged."""
    if dist is None:
        return [float(x) for x in totals]
    import torch
    tt = torch.tensor([float(x) for x in totals], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return [float(x) for x in tt]


def replica_rate(world, units_per_rank, seconds):
    """Whole-job throughput of `world` replicas that each processed
    `units_per_rank` units, the slowest in `seconds`."""
    return world * units_per_rank / seconds


def _timed(step, stream, flush, steps, clocks=None):
    """CUDA-event time (ms) of each of `steps` calls of step() on `stream`,
    L2 flushed (untimed) before each."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        flush.zero_()
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
    stream.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def _stage_ms(lib, ctx, step, flush):
    """Per-stage times of the exact evaluator (median of 3 profiled steps)."""
    lib.cuacd_profile_stages(ctx.handle, 1)
    out = []
    for _ in range(3):
        flush.zero_()
        step()
        arr = (ctypes.c_float * 6)()
        lib.cuacd_stage_times(ctx.handle, ctypes.cast(arr, ctypes.c_void_p))
        out.append(list(arr))
    lib.cuacd_profile_stages(ctx.handle, 0)
    return np.median(np.array(out), axis=0).tolist()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-search", action="store_true", help="skip the whole-search comparison")
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
    from cuacd_b200 import scorer as S
    lib = cuacd_b200._lib
    lib.cuacd_profile_stages.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.cuacd_stage_times.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    dev = local
    torch.cuda.set_device(dev)
    ctx = cuacd_b200.Context(dev)
    sc = S.Scorer.load(ctx)
    v, t = workload()
    planes = planes_for(ctx, v, t)
    n = len(planes)
    hull_vol = S.part_hull_volume(ctx, v)     # every part of the search carries its hull

    # device-resident inputs
    dv = torch.from_numpy(v.reshape(-1)).cuda()
    dt = torch.from_numpy(t.reshape(-1).astype(np.int32)).cuda()
    dp = torch.from_numpy(planes.reshape(-1)).cuda()
    res_bytes = ctypes.sizeof(cuacd_b200.CandResult) * n
    dres = torch.empty(res_bytes, dtype=torch.uint8, device="cuda")
    dres_p = torch.empty(res_bytes, dtype=torch.uint8, device="cuda")
    dpred = torch.empty(n, dtype=torch.float32, device="cuda")
    deval = torch.empty(n, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream(device=dev)
    fn_dev = cuacd_b200._fn("cuacd_eval_candidates_device")
    fn_pdev = cuacd_b200._fn("cuacd_eval_candidates_pruned_device")
    n_eval = ctypes.c_int(0)

    def step():
        rc = fn_dev(ctx.handle, ctypes.c_void_p(dv.data_ptr()), len(v), ctypes.c_void_p(dt.data_ptr()), len(t),
                    ctypes.c_void_p(dp.data_ptr()), n, 1, 2000.0, 1000, 0, ctypes.c_void_p(dres.data_ptr()),
                    ctypes.c_void_p(stream.cuda_stream))
        if rc:
            raise RuntimeError(f"cuacd error {rc}: {lib.gpu_last_error(ctx.handle)}")

    def step_pruned():
        rc = fn_pdev(ctx.handle, sc._h, ctypes.c_void_p(dv.data_ptr()), len(v), ctypes.c_void_p(dt.data_ptr()),
                     len(t), float(hull_vol), ctypes.c_void_p(dp.data_ptr()), n, 1, 2000.0, 1000, 0, TOP_K,
                     float(MARGIN), ctypes.c_void_p(dres_p.data_ptr()), ctypes.c_void_p(dpred.data_ptr()),
                     ctypes.c_void_p(deval.data_ptr()), ctypes.byref(n_eval), ctypes.c_void_p(stream.cuda_stream))
        if rc:
            raise RuntimeError(f"cuacd error {rc}: {lib.gpu_last_error(ctx.handle)}")

    def results(buf):
        host = (cuacd_b200.CandResult * n)()
        hbuf = buf.cpu().numpy()                  # keep the host copy alive for the memmove
        ctypes.memmove(host, hbuf.ctypes.data, res_bytes)
        return host

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        for _ in range(args.warmup):
            step_pruned()
        stream.synchronize()
        # correctness guards on the resident paths
        exact = results(dres)
        pruned = results(dres_p)
        if any(r.err for r in exact) or any(r.err for r in pruned):
            raise RuntimeError("device evaluation reported errors")
        ev_mask = deval.cpu().numpy().astype(bool)
        for i in np.nonzero(ev_mask)[0]:
            if bytes(pruned[i]) != bytes(exact[i]):
                raise RuntimeError(f"pruned result {i} differs from the exact evaluator")
        n_ok = sum(r.ok for r in exact)
        sx = np.array([r.score_full if r.ok else np.inf for r in exact])
        sp = np.array([r.score_full if (r.ok and m) else np.inf for r, m in zip(pruned, ev_mask)])
        quality = {"top_k": TOP_K, "margin": MARGIN, "planes_exact_per_step": int(ev_mask.sum()),
                   "best_exact_score": float(sx.min()), "best_pruned_score": float(sp.min()),
                   "same_best_plane": bool(np.argmin(sp) == np.argmin(sx))}

        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = ctx.launch_count()
        ms_exact = _timed(step, stream, flush, args.steps)
        l1 = ctx.launch_count()
        with Clocks(dev) as clk:
            ms_pruned = _timed(step_pruned, stream, flush, args.steps)
        l2 = ctx.launch_count()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        stage_exact = _stage_ms(lib, ctx, step, flush)
        stage_pruned = _stage_ms(lib, ctx, step_pruned, flush)

    # e2e through the public host-pointer entry points with pinned buffers
    pv = torch.from_numpy(v.reshape(-1)).pin_memory()
    pt = torch.from_numpy(t.reshape(-1).astype(np.int32)).pin_memory()
    pp = torch.from_numpy(planes.reshape(-1)).pin_memory()
    pres = torch.empty(res_bytes, dtype=torch.uint8).pin_memory()
    ppred = torch.empty(n, dtype=torch.float32).pin_memory()
    peval = torch.empty(n, dtype=torch.int32).pin_memory()
    fn_host = cuacd_b200._fn("cuacd_eval_candidates")
    fn_phost = cuacd_b200._fn("cuacd_eval_candidates_pruned")

    def host_step():
        rc = fn_host(ctx.handle, ctypes.c_void_p(pv.data_ptr()), len(v), ctypes.c_void_p(pt.data_ptr()), len(t),
                     ctypes.c_void_p(pp.data_ptr()), n, 1, 2000.0, 1000, 0, ctypes.c_void_p(pres.data_ptr()))
        if rc:
            raise RuntimeError(f"cuacd error {rc}")

    def host_step_pruned():
        rc = fn_phost(ctx.handle, sc._h, ctypes.c_void_p(pv.data_ptr()), len(v), ctypes.c_void_p(pt.data_ptr()),
                      len(t), float(hull_vol), ctypes.c_void_p(pp.data_ptr()), n, 1, 2000.0, 1000, 0, TOP_K,
                      float(MARGIN), ctypes.c_void_p(pres.data_ptr()), ctypes.c_void_p(ppred.data_ptr()),
                      ctypes.c_void_p(peval.data_ptr()), ctypes.byref(n_eval))
        if rc:
            raise RuntimeError(f"cuacd error {rc}")

    def wall(fn):
        for _ in range(args.warmup):
            fn()
        tt = []
        for _ in range(args.steps):
            flush.zero_(); torch.cuda.synchronize()
            t0 = time.perf_counter()
            fn()
            tt.append(time.perf_counter() - t0)
        return sum(tt)

    e2e_exact_s = wall(host_step)
    e2e_s = wall(host_step_pruned)

    tot_ms, tot_exact_ms, e2e_s, e2e_exact_s = replica_max(
        [sum(ms_pruned), sum(ms_exact), e2e_s, e2e_exact_s], dist, "cuda")
    world_n = world
    value = replica_rate(world_n, n * args.steps, tot_ms / 1000.0)
    e2e_val = replica_rate(world_n, n * args.steps, e2e_s)

    # roofline of the dominant stage of the pruned step's exact evaluation
    names = ["k_cut_planes", "hull_pipeline", "k_hd_prep", "k_hd_plan", "k_hd_query", "k_eval_finish"]

    def roofline(stage_ms, res, mask):
        dom = int(np.argmax(stage_ms))
        V, T = len(v), len(t)
        sel = [r for r, m in zip(res, mask) if m]
        k = len(sel)
        Vf = sum(r.nv[0] + r.nv[1] for r in sel); Tf = sum(r.nt[0] + r.nt[1] for r in sel)
        Hv = sum(r.hull_nv[0] + r.hull_nv[1] for r in sel); Ht = sum(r.hull_nt[0] + r.hull_nt[1] for r in sel)
        alg = {
            "k_cut_planes": 12 * (V + T) * k + 12 * (Vf + Tf),
            "hull_pipeline": 12 * (Vf + Tf) + 12 * (Hv + Ht),
            "k_hd_prep": 12 * (Vf + Tf) + 12 * (Hv + Ht),
            "k_hd_plan": 0,
            "k_hd_query": 12 * (Vf + Tf) + 12 * (Hv + Ht),
            "k_eval_finish": 0,
        }
        peak, peak_kind = peaks()
        achieved = alg[names[dom]] / (stage_ms[dom] / 1000.0) / 1e9
        return {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": ncu_traffic(names[dom], k), "ncu_counters": ncu_counters(names[dom]),
                "algorithmic_bytes": int(alg[names[dom]]), "planes": k,
                "stage_ms": {kk: round(x, 4) for kk, x in zip(names, stage_ms)}}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_n, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (exact int/f64 predicates); bf16 network",
            "data": "synthetic", "config": config(n, v, t),
            "candidates_ok": int(n_ok), "gpu_launches": int(l2 - l1), "clocks": clk.summary(),
            "pruning": quality,
            "roofline": roofline(stage_pruned, pruned, ev_mask),
            "e2e": {"value": e2e_val, "unit": UNIT,
                    "h2d_bytes_per_step": int(v.nbytes + t.astype(np.int32).nbytes + planes.nbytes),
                    "d2h_bytes_per_step": int(res_bytes + 8 * n)},
            "exact": {"value": replica_rate(world_n, n * args.steps, tot_exact_ms / 1000.0),
                      "ms_per_step": tot_exact_ms / args.steps, "gpu_launches": int(l1 - l0),
                      "e2e": replica_rate(world_n, n * args.steps, e2e_exact_s),
                      "roofline": roofline(stage_exact, exact, np.ones(n, bool))}}
    if not args.no_search:
        with S.Scorer.load(ctx, S.RV_WEIGHTS_PATH) as rv, S.Scorer(ctx, seed=1) as raw:
            line["search"] = search_leg(ctx, rv, raw)
            line["config4"] = config4_leg(ctx, rv)
    if rank == 0 and world_n == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(v, t, planes)
    if rank == 0:
        print(json.dumps(line), flush=True)
    del sc
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
