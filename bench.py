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
                            "dram_throughput_pct": float(p[7])}
    except (OSError, ValueError):
        pass
    return None


def workloads():
    """The seeded workload generators (cuacd_b200/workloads.py, plain numpy),
    loaded by path: the reference arm must not import the package, whose
    import maps this library's shared object into the process."""
    import importlib.util
    name = "_cuacd_workloads"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "cuacd_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def workload():
    v, t = workloads().candidate_mesh()
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
    W = workloads()
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


def config4_sample():
    return workloads().batch_meshes(512, 500, 200_000, seed=3, select={i for i in range(512) if i % 16 in (0, 5)})


def config4_leg(ctx, scorer):
    """Config 4 sample: the 64 meshes with index 0 or 5 mod 16 of the 512
    uneven synthetic meshes (500 to 200,000 triangles; displaced icospheres
    and unions of 2-6 boxes, seed 3), whole searches with config 4's
    parameters (tau 0.05, width 30/5, depth 2, 16 concave edges), exact and
    pruned; one untimed pass first."""
    meshes = config4_sample()
    kw = dict(width=30, width2=5, depth=2, threshold=0.05, max_iters=100, n_concave_edges=16)
    out = {}
    per_mesh = {}
    for name, extra in (("exact", {}), ("pruned", {"scorer": scorer, "top_k": SEARCH_TOP_K, "beam": SEARCH_BEAM})):
        for v, t in meshes:
            ctx.lookahead_decompose(v, t, **kw, **extra)
        t0 = time.perf_counter()
        parts = [ctx.lookahead_decompose(v, t, **kw, **extra) for v, t in meshes]
        dt = time.perf_counter() - t0
        per_mesh[name] = parts
        out[name] = {"meshes_per_s": len(meshes) / dt, "s": dt, "parts": int(sum(len(p) for p in parts)),
                     "parts_per_mesh": [len(p) for p in parts],
                     "max_rv_cost": float(max(part_cost_max(p) for p in parts))}
    # the same searches as one batch (cuacd_lookahead_decompose_batch): the
    # levels of all 64 meshes share their launches; the parts must be the
    # per-mesh calls' parts
    for name, extra in (("batch_exact", {}),
                        ("batch_pruned", {"scorer": scorer, "top_k": SEARCH_TOP_K, "beam": SEARCH_BEAM})):
        ctx.lookahead_decompose_batch(meshes[:8], **kw, **extra)
        t0 = time.perf_counter()
        parts = ctx.lookahead_decompose_batch(meshes, **kw, **extra)
        dt = time.perf_counter() - t0
        ref = per_mesh[name.split("_")[1]]
        same = all(len(a) == len(b) and all(np.array_equal(x, y) for pa, pb in zip(a, b) for x, y in zip(pa, pb))
                   for a, b in zip(parts, ref))
        out[name] = {"meshes_per_s": len(meshes) / dt, "s": dt, "parts": int(sum(len(p) for p in parts)),
                     "same_parts_as_per_mesh_calls": bool(same), "stats": list(ctx.last_search_stats),
                     "max_rv_cost": float(max(part_cost_max(p) for p in parts))}
    out["workload"] = (f"config 4 sample: {len(meshes)} of the 512 meshes (index 0 or 5 mod 16), "
                       f"{min(len(t) for _, t in meshes)}-{max(len(t) for _, t in meshes)} tris")
    return out


def remesh_leg(ctx, args, cpu_baseline=True):
    """Remesh front end (Context.preprocess): the 40,960-triangle ridged
    sphere of the headline workload at resolutions 64 and 128, through the
    public call (host arrays in and out), mean wall time over `steps` calls
    after `warmup`; the output's triangle count and GPU audit verdict (0:
    watertight, manifold, oriented)."""
    v, t = workload()
    out = {"workload": f"{len(t):,}-triangle sphere (config 3 mesh)"}
    for R in (64, 128):
        for _ in range(max(1, args.warmup)):
            ctx.preprocess(v, t, resolution=R)
        l0 = ctx.launch_count()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            rv, rt = ctx.preprocess(v, t, resolution=R)
        dt = (time.perf_counter() - t0) / args.steps
        out[f"R{R}"] = {"ms_per_call": dt * 1e3, "in_tris_per_s": len(t) / dt, "out_tris": int(len(rt)),
                        "out_verts": int(len(rv)), "gpu_launches_per_call": (ctx.launch_count() - l0) / args.steps,
                        "audit_flags": int(ctx.check_mesh(rv, rt)["flags"])}
    if cpu_baseline and not args.no_cpu_baseline:
        from oracle import remesh as RMO                    # the CPU restatement, timed as the baseline
        t0 = time.perf_counter()
        ov, ot = RMO.remesh(v, t, 64)
        dt = time.perf_counter() - t0
        gv, gt = ctx.preprocess(v, t, resolution=64)
        out["cpu_baseline"] = {"value": dt * 1e3, "unit": "ms per call", "cores": 1, "kind": "port",
                               "sample": "one call at R = 64 (numpy restatement)",
                               "same_output": bool(np.array_equal(ov, gv) and np.array_equal(ot, gt))}
    return out


def oracle_planes(v, t):
    """The same 30 planes as the library's GPU generator, from the oracle
    (the GPU path is bit-exact to it)."""
    from oracle import oracle as O
    return np.ascontiguousarray(np.concatenate(
        [O.concave_planes(v, t, 16, 0.005, 3.49)[:N_EDGE],
         np.stack([O.axis_plane(v, WIDTH, i, 0.0125) for i in range(WIDTH)])]).astype(np.float32))


def cpu_baseline(v, t, planes, budget_s=20.0):
    """Oracle port on all host cores over a bounded sample of the workload:
    whole 30-plane steps until about budget_s/2 seconds have passed."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    done = 0
    while True:
        O.eval_candidates(v, t, planes, hausdorff=True, threads=cores)
        done += len(planes)
        if time.perf_counter() - t0 > budget_s * 0.5 or done >= 4 * len(planes):
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{done} candidates ({len(planes)} planes per step) of the same workload, "
                      f"oracle (FP64/exact C) with {cores} threads"}


def cpu_hull_baseline(clouds, budget_s=10.0):
    """Oracle hulls (exact int64 on the quantised grid) of the config-1
    clouds on all host cores (one cloud per thread; ctypes releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    done = 0
    with ThreadPoolExecutor(cores) as ex:
        while True:
            list(ex.map(O.hull, clouds))
            done += len(clouds)
            if time.perf_counter() - t0 > budget_s * 0.5:
                break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "clouds/s", "cores": cores, "kind": "port",
            "sample": f"{done} clouds of 1,000 points (the config-1 batch, whole passes), oracle with {cores} threads"}


def cpu_hausdorff_baseline(a, b, total=20000):
    """Oracle Hausdorff (FP64, brute force nearest triangle) of the config-2
    pair on all host cores, `total` samples per direction."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    O.hausdorff(*a, *b, total=total, threads=cores)
    dt = time.perf_counter() - t0
    return {"value": 2 * total / dt, "unit": "samples/s", "cores": cores, "kind": "port",
            "sample": f"{total} samples per direction (of the 10^6 of a step), oracle with {cores} threads"}


def run_reference(args, rank, world):
    """The reference arm.  The reference implements this path only in CUDA
    (its CPU baselines need sources absent from its tree), so the line's
    value is the oracle port of the path (the reference's algorithm in
    FP64/exact C) on all host cores, on the same 30 planes of the same mesh.
    The reference's own GPU path, built unmodified from its sources into
    oracle/_ref, is timed beside it in a child process (its own extension
    loaded, nothing of this library) under "reference_gpu"."""
    if rank != 0:
        return
    from oracle import oracle as O
    v, t = workload()
    planes = oracle_planes(v, t)
    n = len(planes)
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        O.eval_candidates(v, t, planes, hausdorff=True, threads=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.eval_candidates(v, t, planes, hausdorff=True, threads=cores)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    val = n * args.steps / total
    line = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(n, v, t), "impl": "reference",
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"all {n} planes per step, oracle with {cores} threads"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_reference_gpu:
        line["reference_gpu"] = reference_gpu(args)
    print(json.dumps(line), flush=True)


REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def reference_gpu(args):
    """Run the reference's GPU legs in a child process; its JSON or why not."""
    if not os.path.exists(os.path.join(REF_DIR, "_gpu.so")):
        return {"unavailable": "the reference's GPU build (oracle/_ref) is absent"}
    cmd = [sys.executable, os.path.abspath(__file__), "--ref-gpu-child", "--steps", str(args.steps),
           "--warmup", str(args.warmup)]
    if args.no_search:
        cmd.append("--no-search")
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    except subprocess.TimeoutExpired:
        return {"unavailable": "the reference's GPU legs ran past 600 s"}
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"unavailable": f"reference GPU child exited {r.returncode}: {r.stderr.strip()[-300:]}"}
    return json.loads(lines[-1])


def load_ref_gpu():
    """The reference's CPython extension (oracle/_ref/_gpu.so) with its
    fatbin, initialised on device 0 as its Python wrapper does."""
    import importlib.machinery
    import importlib.util
    loader = importlib.machinery.ExtensionFileLoader("_gpu", os.path.join(REF_DIR, "_gpu.so"))
    spec = importlib.util.spec_from_loader("_gpu", loader)
    g = importlib.util.module_from_spec(spec)
    loader.exec_module(g)
    with open(os.path.join(REF_DIR, "kernels.fatbin"), "rb") as f:
        g.set_fatbin(f.read())
    g.init(0, 0)
    return g


def _ref_hull_call(g, clouds, kdop):
    """One call of the reference's hull entry point over a batch of clouds,
    with the output caps its wrapper uses (cuacd/__init__.py:203-205,289-290)."""
    n = len(clouds)
    packed = np.ascontiguousarray(np.concatenate(clouds), np.float32)
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
    out = []
    for i in range(n):
        hv = ov[i * mhv * 3:(i * mhv + onv[i]) * 3].reshape(-1, 3)
        ht = ot[i * mht * 3:(i * mht + ont[i]) * 3].reshape(-1, 3)
        out.append((hv, ht, float(ovol[i])))
    return out, err


def _fp32_volume(v, t):
    """The reference wrapper's host-side hull volume (cuacd/__init__.py:222-231)."""
    a, b, c = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    return abs(float(np.einsum("ij,ij->i", a, np.cross(b, c)).sum()) / 6.0)


def _ref_eval_candidate(g, v, t, p, caps):
    """One candidate through the reference's GPU entry points, the steps of
    its la_expand/la_hull (cuda/la_expand.cu:65-424) plus the per-part
    Hausdorff the full score needs: the cut with caps (test_plane_cut), the
    k-DOP hull and volume of both fragments (one kdop_hull call), both
    fragments' volumes (one batch_mesh_volume call), and the Hausdorff
    distance of each fragment to its hull (two test_hausdorff calls)."""
    pv, pt, nvv, ntt, vcap, tcap = caps
    a, b, c, d = (float(x) for x in p)
    n_pv, n_pt, n_nv, n_nt = g.test_plane_cut(v.ctypes.data, len(v), t.ctypes.data, len(t), a, b, c, d,
                                              pv.ctypes.data, vcap, pt.ctypes.data, tcap,
                                              nvv.ctypes.data, vcap, ntt.ctypes.data, tcap)
    if n_pt == 0 or n_nt == 0:
        return False
    frags = [(pv[:3 * n_pv].reshape(-1, 3), pt[:3 * n_pt].reshape(-1, 3)),
             (nvv[:3 * n_nv].reshape(-1, 3), ntt[:3 * n_nt].reshape(-1, 3))]
    hulls, _ = _ref_hull_call(g, [f[0] for f in frags], kdop=True)
    allv = np.ascontiguousarray(np.concatenate([f[0] for f in frags]))
    allt = np.ascontiguousarray(np.concatenate([f[1] for f in frags]))
    toff = np.array([0, n_pt, n_pt + n_nt], np.int32)
    voff = np.array([0, n_pv, n_pv + n_nv], np.int32)
    vols = np.empty(2, np.float32)
    g.batch_mesh_volume(allv.ctypes.data, len(allv), allt.ctypes.data, len(allt), toff.ctypes.data,
                        voff.ctypes.data, 2, vols.ctypes.data)
    out = np.zeros(1, np.float32)
    for (fv, ft), (hv, ht, _) in zip(frags, hulls):
        fv, ft = np.ascontiguousarray(fv), np.ascontiguousarray(ft)
        hv, ht = np.ascontiguousarray(hv), np.ascontiguousarray(ht)
        g.test_hausdorff(hv.ctypes.data, len(hv), ht.ctypes.data, len(ht), fv.ctypes.data, len(fv),
                         ft.ctypes.data, len(ft), out.ctypes.data)
    return True


def _ref_lookahead(g, v, t, n_edges):
    """The reference's lookahead_decompose as its Python wrapper drives it
    (cuacd/__init__.py:367-454): scipy hull of the input with outward
    winding, then the extension call; returns the parts as arrays."""
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
    raw = g.lookahead_decompose(v.ctypes.data, len(v), t.ctypes.data, len(t), hv.ctypes.data, len(hv),
                                ht.ctypes.data, len(ht), 100, 30, 5, 0.05, 2, 0, 16, 0, 0,
                                n_concave_edges=n_edges)
    parts = []
    for vb, tb, nv, nt, hvb, htb, hnv, hnt, _, _ in raw:
        parts.append((np.frombuffer(vb, np.float32).reshape(nv, 3), np.frombuffer(tb, np.int32).reshape(nt, 3),
                      np.frombuffer(hvb, np.float32).reshape(hnv, 3), np.frombuffer(htb, np.int32).reshape(hnt, 3)))
    return parts


def ref_gpu_child(args):
    """The reference's own GPU path (built unmodified from its sources) on
    the bench's workloads, through its CPython extension, wall clock per
    call as its synchronous entry points return.  Prints one JSON line."""
    from oracle import oracle as O
    W = workloads()
    g = load_ref_gpu()
    out = {"build": "eliphatfs/cuacd sources, nvcc -O3 --use_fast_math sm_100 (its setup.py flags), "
                    "run through its _gpu extension"}
    # config 3: 30 candidates per step
    v, t = workload()
    v = np.ascontiguousarray(v, np.float32)
    t = np.ascontiguousarray(t, np.int32)
    planes = oracle_planes(v, t)
    vcap, tcap = len(v) + 2 * len(t), 3 * len(t) + 64
    caps = (np.empty(vcap * 3, np.float32), np.empty(tcap * 3, np.int32), np.empty(vcap * 3, np.float32),
            np.empty(tcap * 3, np.int32), vcap, tcap)
    for _ in range(args.warmup):
        for p in planes:
            _ref_eval_candidate(g, v, t, p, caps)
    with Clocks(0) as clk:
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            ok = sum(_ref_eval_candidate(g, v, t, p, caps) for p in planes)
            times.append(time.perf_counter() - t0)
    out["config3"] = {"value": len(planes) * args.steps / sum(times), "unit": UNIT,
                      "ms_per_step": 1000 * sum(times) / args.steps, "candidates_ok": int(ok),
                      "steps": args.steps, "warmup": args.warmup, "clocks": clk.summary(),
                      "workload": "the same 30 planes of the 40,960-tri sphere; per candidate test_plane_cut + "
                                  "kdop_hull (both fragments) + batch_mesh_volume + 2 test_hausdorff"}
    # config 1: 256 x 1,000-point clouds, batch_hull_volume's steps
    clouds = W.hull_clouds(256, 1000, 0)
    def c1():
        hulls, _ = _ref_hull_call(g, clouds, kdop=False)
        return [_fp32_volume(hv, ht) for hv, ht, _ in hulls]
    for _ in range(args.warmup):
        c1()
    with Clocks(0) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            c1()
        dt = time.perf_counter() - t0
    out["config1"] = {"value": len(clouds) * args.steps / dt, "unit": "clouds/s", "ms_per_step": 1000 * dt / args.steps,
                      "clocks": clk.summary(),
                      "workload": "256 x 1,000 uniform points (seed 0): hull_dandc + FP32 host volumes, "
                                  "as its batch_hull_volume"}
    # config 2: the 20,480-tri sphere against its hull, at the reference's
    # own sample rule (HD_RESOLUTION 2000 is a plain #define in its source)
    sv, st = W.hausdorff_sphere(level=5)
    (hv, ht, _), = _ref_hull_call(g, [sv], kdop=False)[0]
    hv, ht = np.ascontiguousarray(hv), np.ascontiguousarray(ht)
    sv, st = np.ascontiguousarray(sv, np.float32), np.ascontiguousarray(st, np.int32)
    n_samp = O.hd_sample_count(hv, ht) + O.hd_sample_count(sv, st)
    res = np.zeros(1, np.float32)
    def c2():
        g.test_hausdorff(hv.ctypes.data, len(hv), ht.ctypes.data, len(ht), sv.ctypes.data, len(sv),
                         st.ctypes.data, len(st), res.ctypes.data)
    for _ in range(args.warmup):
        c2()
    with Clocks(0) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            c2()
        dt = time.perf_counter() - t0
    out["config2"] = {"value": n_samp * args.steps / dt, "unit": "samples/s", "ms_per_step": 1000 * dt / args.steps,
                      "samples_per_step": int(n_samp), "hausdorff": float(res[0]), "clocks": clk.summary(),
                      "workload": "20,480-tri displaced icosphere (seed 1) vs its hull, both directions, "
                                  "the reference's 2000-per-unit-area rule (its resolution is fixed in source)"}
    if not args.no_search:
        meshes = config4_sample()
        for vv, tt in meshes[:4]:                    # untimed: the pools grow
            _ref_lookahead(g, vv, tt, 16)
        with Clocks(0) as clk:
            t0 = time.perf_counter()
            parts = [_ref_lookahead(g, vv, tt, 16) for vv, tt in meshes]
            dt = time.perf_counter() - t0
        out["config4"] = {"meshes_per_s": len(meshes) / dt, "s": dt, "parts": int(sum(len(p) for p in parts)),
                          "parts_per_mesh": [len(p) for p in parts],
                          "max_rv_cost": float(max(part_cost_max(p) for p in parts)), "clocks": clk.summary(),
                          "workload": "the 64-mesh config-4 sample, tau 0.05, width 30/5, depth 2, 16 concave edges"}
    g.destroy()
    print(json.dumps(out), flush=True)


def config1_leg(ctx, stream, flush, args):
    """Config 1: exact hulls and volumes of 256 clouds x 1,000 uniform points
    (seed 0) in one batch.  value: device-resident (cuacd_hull_batch_device,
    inputs in HBM), CUDA events, L2 flushed before each step; e2e: the public
    Context.batch_hull_volume with host arrays."""
    import torch
    import cuacd_b200
    W = workloads()
    clouds = W.hull_clouds(256, 1000, 0)
    n, k = len(clouds), 1000
    packed = np.ascontiguousarray(np.concatenate(clouds), np.float32)
    off = np.arange(0, n * k + 1, k, dtype=np.int32)
    mht = 2 * k - 4
    d_pts = torch.from_numpy(packed.reshape(-1)).cuda()
    d_off = torch.from_numpy(off).cuda()
    d_v = torch.empty(n * k * 3, dtype=torch.float32, device="cuda")
    d_t = torch.empty(n * mht * 3, dtype=torch.int32, device="cuda")
    d_nv, d_nt, d_err = (torch.empty(n, dtype=torch.int32, device="cuda") for _ in range(3))
    d_vol = torch.empty(n, dtype=torch.float32, device="cuda")
    fn = cuacd_b200._fn("cuacd_hull_batch_device")
    P = lambda x: ctypes.c_void_p(x.data_ptr())

    def step():
        rc = fn(ctx.handle, P(d_pts), P(d_off), n, k, k, mht, P(d_v), P(d_t), P(d_nv), P(d_nt), P(d_vol), P(d_err),
                ctypes.c_void_p(stream.cuda_stream))
        if rc:
            raise RuntimeError(f"cuacd error {rc}")

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        stream.synchronize()
        if int(d_err.abs().sum()):
            raise RuntimeError("config 1: hull errors")
        l0 = ctx.launch_count()
        ms = _timed(step, stream, flush, args.steps)
        launches = ctx.launch_count() - l0
    nv, nt = int(d_nv.sum()), int(d_nt.sum())
    vols = d_vol.cpu().numpy()

    def e2e():
        ctx.batch_hull_volume(clouds)
    for _ in range(args.warmup):
        e2e()
    tt = []
    for _ in range(args.steps):
        flush.zero_(); torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e()
        tt.append(time.perf_counter() - t0)
    alg = 12 * n * k + 12 * (nv + nt)
    avg = sum(ms) / len(ms)
    peak, peak_kind = peaks()
    achieved = alg / (avg / 1000.0) / 1e9
    out = {"value": n * args.steps / (sum(ms) / 1000.0), "unit": "clouds/s", "ms_per_step": avg,
           "gpu_launches": int(launches),
           "workload": "config1: 256 clouds x 1,000 float32 points uniform in [-1,1]^3 (seed 0), "
                       "exact hull index sets + volumes, one batch per step",
           "hull_verts": nv, "hull_tris": nt, "volume_sum": float(vols.sum()),
           "roofline": {"bound": "hbm", "kernel": "hull_pipeline", "achieved": achieved, "peak": peak,
                        "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                        "traffic": ncu_traffic("config1_hull", n), "algorithmic_bytes": int(alg)},
           "e2e": {"value": n * args.steps / sum(tt), "unit": "clouds/s",
                   "h2d_bytes_per_step": int(packed.nbytes + off.nbytes), "d2h_bytes_per_step": int(16 * n)}}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_hull_baseline(clouds)
    return out


C2_SAMPLES = 10 ** 6


def config2_leg(ctx, stream, flush, args):
    """Config 2: sampled Hausdorff distance between the 20,480-triangle
    displaced icosphere (seed 1) and its exact hull, 10^6 samples per
    surface per direction.  value: device-resident
    (cuacd_hausdorff_batch_device), samples/s over both directions, CUDA
    events, L2 flushed; e2e: Context.hausdorff with host arrays.  Also timed
    at the reference's own sample rule (2000 per unit area, min 1000)."""
    import torch
    import cuacd_b200
    W = workloads()
    sv, st = W.hausdorff_sphere(level=5)
    (hv, ht, _), = ctx.batch_hull_dandc_mesh([sv])
    a = (np.ascontiguousarray(hv, np.float32), np.ascontiguousarray(ht, np.int32))
    b = (np.ascontiguousarray(sv, np.float32), np.ascontiguousarray(st, np.int32))
    dav, dat = torch.from_numpy(a[0].reshape(-1)).cuda(), torch.from_numpy(a[1].reshape(-1)).cuda()
    dbv, dbt = torch.from_numpy(b[0].reshape(-1)).cuda(), torch.from_numpy(b[1].reshape(-1)).cuda()
    avo = np.array([0, len(a[0])], np.int32); ato = np.array([0, len(a[1])], np.int32)
    bvo = np.array([0, len(b[0])], np.int32); bto = np.array([0, len(b[1])], np.int32)
    d_out = torch.zeros(1, dtype=torch.float32, device="cuda")
    fn = cuacd_b200._fn("cuacd_hausdorff_batch_device")
    P = lambda x: ctypes.c_void_p(x.data_ptr())
    H = lambda x: ctypes.c_void_p(x.ctypes.data)

    def run(total):
        def step():
            rc = fn(ctx.handle, 1, P(dav), H(avo), P(dat), H(ato), P(dbv), H(bvo), P(dbt), H(bto),
                    2000.0, 1000, total, P(d_out), ctypes.c_void_p(stream.cuda_stream))
            if rc:
                raise RuntimeError(f"cuacd error {rc}")
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                step()
            stream.synchronize()
            l0 = ctx.launch_count()
            ms = _timed(step, stream, flush, args.steps)
            return ms, ctx.launch_count() - l0, float(d_out.item())

    ms, launches, h = run(C2_SAMPLES)
    n_samp = 2 * C2_SAMPLES
    ms_rule, _, h_rule = run(0)

    def e2e():
        ctx.hausdorff(*a, *b, total=C2_SAMPLES)
    for _ in range(args.warmup):
        e2e()
    tt = []
    for _ in range(args.steps):
        flush.zero_(); torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e()
        tt.append(time.perf_counter() - t0)
    avg = sum(ms) / len(ms)
    alg = 12 * (len(a[0]) + len(a[1]) + len(b[0]) + len(b[1]))
    peak, peak_kind = peaks()
    achieved = alg / (avg / 1000.0) / 1e9
    out = {"value": n_samp * args.steps / (sum(ms) / 1000.0), "unit": "samples/s", "ms_per_step": avg,
           "gpu_launches": int(launches), "hausdorff": h,
           "workload": "config2: 20,480-tri displaced icosphere (radius 1+0.25*sum of 8 sines, seed 1) vs its "
                       "exact hull, 10^6 samples per surface, both directions",
           "roofline": {"bound": "hbm", "kernel": "k_hd_prep+k_hd_query", "achieved": achieved, "peak": peak,
                        "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                        "traffic": None, "algorithmic_bytes": int(alg),
                        "note": "the samples are generated on chip: the meshes are the only bytes, so the "
                                "query is issue/latency-bound, not HBM-bound"},
           "e2e": {"value": n_samp * args.steps / sum(tt), "unit": "samples/s",
                   "h2d_bytes_per_step": int(sum(x.nbytes for x in a + b)), "d2h_bytes_per_step": 4},
           "reference_rule": {"ms_per_step": sum(ms_rule) / len(ms_rule), "hausdorff": h_rule,
                              "note": "2000 samples per unit area, min 1000 (cuda/hausdorff.cuh:380-382)"}}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_hausdorff_baseline(a, b)
    return out


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


# ---------------------------------------------------------------------------
# Side-by-side legs against the reference's own GPU build (oracle/_ref, built
# from the reference's sources by oracle/Makefile.ref): `python bench.py
# --compare NAME --out OUT.json`.  Each loads the reference's CPython
# extension the way its Python wrapper does, times its public calls and this
# library's on the same seeded inputs, and writes one JSON file.  They are
# measurements for the profiles, not part of the timed benchmark line.
# ---------------------------------------------------------------------------

SEARCH_KW = dict(max_iters=100, width=30, width2=5, threshold=0.05, depth=2, quick_depth=0, max_n_cutting=16)


def _ref_module():
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_ref_gpu as MR
    return MR


def compare_search(out_path, full=False):
    """Whole lookahead searches: the reference (cuacd/__init__.py:367-454:
    scipy hull of the input with outward winding, then
    `_gpu.lookahead_decompose`) beside this library's exact and pruned
    searches, on the six ridged spheres (32 concave edges) and the config-4
    sample (or, with --full, all 512 meshes; 16 concave edges).  Per mesh:
    triangles, parts, seconds, largest part rv cost; one untimed pass over
    the six spheres first in every mode."""
    MR = _ref_module()
    W = workloads()
    S = {"search": (search_meshes(), 32)}
    if full:
        S["config4_full"] = (W.batch_meshes(512, 500, 200_000, seed=3), 16)
    else:
        S["config4"] = (config4_sample(), 16)
    kw = SEARCH_KW

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
                                    ht.ctypes.data, len(ht), kw["max_iters"], kw["width"], kw["width2"],
                                    kw["threshold"], kw["depth"], kw["quick_depth"], kw["max_n_cutting"], 0, 0,
                                    n_concave_edges=n_edges)
        dt = time.perf_counter() - t0
        parts = [(np.frombuffer(vb, np.float32).reshape(nv, 3), np.frombuffer(tb, np.int32).reshape(nt, 3),
                  np.frombuffer(hvb, np.float32).reshape(hnv, 3), np.frombuffer(htb, np.int32).reshape(hnt, 3))
                 for vb, tb, nv, nt, hvb, htb, hnv, hnt, _, _ in raw]
        return parts, dt

    def row(t, parts, dt):
        return {"tris": int(len(t)), "parts": len(parts), "s": dt, "max_rv": part_cost_max(parts)}

    rec = {"settings": {**kw, "n_concave_edges": {k: e for k, (_, e) in S.items()}}}
    g = MR.load_ref()
    for v, t in S["search"][0]:
        ref_search(g, v, t, 32)
    for name, (meshes, ne) in S.items():
        rows = []
        for v, t in meshes:
            try:
                parts, dt = ref_search(g, v, t, ne)
                rows.append(row(t, parts, dt))
            except Exception as e:                        # a failed search is recorded
                rows.append({"tris": int(len(t)), "parts": 0, "s": 0.0, "max_rv": 0.0, "error": str(e)[:200]})
        rec[f"reference_{name}"] = rows
        print("reference", name, sum(r["s"] for r in rows), "s", sum(r["parts"] for r in rows), "parts", flush=True)
    g.destroy()
    import cuacd_b200
    from cuacd_b200 import scorer as SC
    with cuacd_b200.Context(0) as ctx, SC.Scorer.load(ctx, SC.RV_WEIGHTS_PATH) as rv:
        for mname, extra in (("exact", {}), ("pruned", {"scorer": rv, "top_k": SEARCH_TOP_K, "beam": SEARCH_BEAM})):
            for v, t in S["search"][0]:
                ctx.lookahead_decompose(v, t, **kw, n_concave_edges=32, **extra)
            for name, (meshes, ne) in S.items():
                rows = []
                for v, t in meshes:
                    t0 = time.perf_counter()
                    try:
                        parts = ctx.lookahead_decompose(v, t, **kw, n_concave_edges=ne, **extra)
                        rows.append(row(t, parts, time.perf_counter() - t0))
                    except RuntimeError as e:
                        rows.append({"tris": int(len(t)), "parts": 0, "s": 0.0, "max_rv": 0.0, "error": str(e)[:200]})
                rec[f"{mname}_{name}"] = rows
                print(mname, name, sum(r["s"] for r in rows), "s", sum(r["parts"] for r in rows), "parts", flush=True)
    with open(out_path, "w") as f:
        json.dump(rec, f)


def compare_hull_sweep(out_path):
    """Batched hull volumes over the shapes of the reference's arena sweep
    (docs/arena_sweep.md: 10000x20, 1000x200, 100x2000, 10x20000 points;
    sphere shell, cube interior, gaussian; seeded).  Reference: its
    `Context.batch_hull_volume` steps (cuacd/__init__.py:185-233: pack,
    `_gpu.hull_dandc` with caps n / 2n-4, FP32 volumes on the host), the
    call alone and the whole method; this library: `batch_hull_volume`.
    Wall clock, median of 5 after a warm-up; hull index sets compared."""
    import statistics
    MR = _ref_module()
    shapes = [(10000, 20), (1000, 200), (100, 2000), (10, 20000)]
    dists = ["sphere_shell", "cube_interior", "gaussian"]

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

    def ref_call(g, cl):
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

    cases = [(n, k, d, 100 + 10 * si + di) for si, (n, k) in enumerate(shapes) for di, d in enumerate(dists)]
    data = {c: clouds(*c) for c in cases}
    rows = {c: {"clouds": c[0], "points": c[1], "dist": c[2]} for c in cases}
    g = MR.load_ref()
    for c in cases:
        cl = data[c]
        ref_call(g, cl)
        calls, whole = [], []
        for _ in range(5):
            t0 = time.perf_counter()
            vols, err, t_call, meshes = ref_call(g, cl)
            whole.append(time.perf_counter() - t0)
            calls.append(t_call)
        rows[c].update(ref_call_ms=1e3 * statistics.median(calls), ref_method_ms=1e3 * statistics.median(whole),
                       ref_errors=int((err != 0).sum()))
        rows[c]["_sets"] = [set(MR.index_set(x, m).tolist()) for x, m in zip(cl, meshes)]
        rows[c]["_vol"] = vols
        print("reference", c[:3], round(rows[c]["ref_call_ms"], 2), "ms", flush=True)
    g.destroy()
    import cuacd_b200
    with cuacd_b200.Context(0) as ctx:
        for c in cases:
            cl = data[c]
            ctx.batch_hull_volume(cl)
            ts = []
            for _ in range(5):
                t0 = time.perf_counter()
                vols, err = ctx.batch_hull_volume(cl)
                ts.append(time.perf_counter() - t0)
            r = rows[c]
            r["ours_ms"] = 1e3 * statistics.median(ts)
            r["ours_errors"] = int((err != 0).sum())
            ours = [set(MR.index_set(x, m[0]).tolist()) for x, m in zip(cl, ctx.batch_hull_dandc_mesh(cl))]
            r["sets_differing"] = int(sum(a != b for a, b in zip(ours, r.pop("_sets"))))
            rv = r.pop("_vol")
            r["max_rel_vol_diff"] = float(np.max(np.abs(vols - rv) / np.maximum(np.abs(rv), 1e-30)))
            r["speedup_vs_ref_method"] = r["ref_method_ms"] / r["ours_ms"]
            print("ours", c[:3], round(r["ours_ms"], 2), "ms, sets differing", r["sets_differing"], flush=True)
    with open(out_path, "w") as f:
        json.dump(list(rows.values()), f)


def compare_hausdorff(out_path):
    """The reference's Hausdorff benchmark (bench/hausdorff_bench.cu, built
    into oracle/_ref/hausdorff_bench; GPU rows, `hausdorff_block`, one block
    per pair: the bunny and the 49160 mesh against their hulls, batches 1 and
    100, CUDA events, 2 warm-up and 5 timed launches) beside
    `cuacd_hausdorff_batch_device` on the same meshes (extracted from the
    benchmark's data header), batches and sampling, meshes resident, CUDA
    events on the call's stream, 2 warm-up and 5 timed calls (mean)."""
    import statistics
    import torch
    r = subprocess.run([os.path.join(REF_DIR, "hausdorff_bench")], capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    lines = [l.split(",") for l in r.stdout.splitlines() if l.strip()]
    ref = [x for x in (dict(zip(lines[0], l)) for l in lines[1:]) if x["algorithm"] == "hausdorff_block"]
    import cuacd_b200
    fn = cuacd_b200._fn("cuacd_hausdorff_batch_device")
    data = np.load(os.path.join(REF_DIR, "hausdorff_bench_data.npz"))
    sets = {"bunny": "BUNNY", "49160": "STL"}
    P = ctypes.c_void_p
    rows = []
    with cuacd_b200.Context(0) as ctx:
        for x in ref:
            k, batch = sets[x["dataset"]], int(x["batch"])
            mv, mt, hv, ht = (data[f"{k}_{n}"] for n in ("verts", "tris", "hull_verts", "hull_tris"))
            dev = [torch.from_numpy(np.ascontiguousarray(np.tile(a, (batch, 1)), dt)).cuda()
                   for a, dt in ((mv, np.float32), (mt, np.int32), (hv, np.float32), (ht, np.int32))]
            offs = [np.arange(batch + 1, dtype=np.int32) * len(a) for a in (mv, mt, hv, ht)]
            out = torch.zeros(batch, dtype=torch.float32, device="cuda")
            stream = torch.cuda.Stream()

            def call():
                rc = fn(ctx.handle, batch, P(dev[0].data_ptr()), P(offs[0].ctypes.data), P(dev[1].data_ptr()),
                        P(offs[1].ctypes.data), P(dev[2].data_ptr()), P(offs[2].ctypes.data), P(dev[3].data_ptr()),
                        P(offs[3].ctypes.data), 2000.0, 1000, 0, P(out.data_ptr()), P(stream.cuda_stream))
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
            m = statistics.mean(ms)
            rows.append({"dataset": x["dataset"], "batch": batch, "ref_ms": float(x["mean_ms"]),
                         "ref_std_ms": float(x["std_ms"]), "ref_dist": float(x["mean_dist"]), "ours_ms": m,
                         "ours_std_ms": statistics.pstdev(ms), "ours_dist": float(d.mean()),
                         "ours_dist_spread": float(d.max() - d.min()), "speedup": float(x["mean_ms"]) / m})
            print(rows[-1], flush=True)
    with open(out_path, "w") as f:
        json.dump(rows, f)


def compare_heap(out_path):
    """Device allocation throughput: the reference's heap benchmark
    (bench/malloc_test_bench.cu, built into oracle/_ref/malloc_test_bench;
    its own heap and CUDA's device malloc/free) at 256 alloc-free iterations
    per block instead of 1,024, so that this library's arena, which frees by
    whole-arena reset, holds a run (1,024 blocks x 256 x 62 KB mean = 16 GB);
    beside `cuacd_arena_bench` on the same workload (thread 0 of each block
    drawing log-uniform sizes in [4 KiB, 256 KiB] into 16 slots), the arena
    reset before each run.  CUDA events, 2 warm-up and 5 timed runs."""
    iters, slots, smin, smax = 256, 16, 4096, 262144
    r = subprocess.run([os.path.join(REF_DIR, "malloc_test_bench"), "--iters", str(iters), "--slots", str(slots),
                        "--size-min", str(smin), "--size-max", str(smax), "--impl", "both"],
                       capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    lines = [l.split(",") for l in r.stdout.splitlines() if l.strip()]
    ref = [dict(zip(lines[0], l)) for l in lines[1:]]
    import cuacd_b200
    fn = cuacd_b200._lib.cuacd_arena_bench
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_uint,
                   ctypes.c_ulonglong, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                   ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)]
    ours = []
    with cuacd_b200.Context(0) as ctx:
        for grid in (1, 4, 16, 64, 256, 1024):
            m, s, fl = ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
            rc = fn(ctx.handle, grid, iters, slots, smin, smax, 20 << 30, 2, 5, ctypes.byref(m), ctypes.byref(s),
                    ctypes.byref(fl))
            if rc:
                raise RuntimeError(f"cuacd error {rc}")
            ours.append({"grid": grid, "mean_ms": m.value, "std_ms": s.value, "failed_allocs": fl.value,
                         "mops": grid * iters / (m.value * 1e-3) / 1e6})
            print(ours[-1], flush=True)
    with open(out_path, "w") as f:
        json.dump({"iters": iters, "slots": slots, "size_min": smin, "size_max": smax, "reference": ref,
                   "reference_log": r.stderr[-1000:], "ours": ours}, f)


def compare_audit(out_path):
    """Mesh audit: the reference's `_gpu.mesh_audit` (one 256-thread block
    per mesh) beside `Context.check_mesh`, on the 40,960- and 327,680-
    triangle spheres; wall clock of the public call, median of 5 after a
    warm-up."""
    import statistics
    MR = _ref_module()
    W = workloads()
    big = [m for m in config4_sample() if len(m[1]) == 327680][0]
    ms = [(n, np.ascontiguousarray(v, np.float32), np.ascontiguousarray(t, np.int32))
          for n, v, t in (("40,960-tri sphere", *W.candidate_mesh()), ("327,680-tri sphere", *big))]

    def timed(fn):
        fn()
        ts = []
        for _ in range(5):
            t0 = time.perf_counter()
            r = fn()
            ts.append(time.perf_counter() - t0)
        return 1e3 * statistics.median(ts), r

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


COMPARE = {"search": compare_search, "hull_sweep": compare_hull_sweep, "hausdorff": compare_hausdorff,
           "heap": compare_heap, "audit": compare_audit}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-search", action="store_true", help="skip the whole-search comparison")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm: skip the reference's own GPU legs")
    ap.add_argument("--ref-gpu-child", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--compare", choices=sorted(COMPARE),
                    help="side-by-side leg against the reference's own GPU build (writes --out)")
    ap.add_argument("--out", help="JSON output of --compare")
    ap.add_argument("--full", action="store_true", help="--compare search: all 512 config-4 meshes")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.ref_gpu_child:
        ref_gpu_child(args)
        return
    if args.compare:
        if not args.out:
            ap.error("--compare needs --out")
        if args.compare == "search":
            compare_search(args.out, full=args.full)
        else:
            COMPARE[args.compare](args.out)
        return

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
    line["config1"] = config1_leg(ctx, stream, flush, args)
    line["config2"] = config2_leg(ctx, stream, flush, args)
    try:
        line["remesh"] = remesh_leg(ctx, args, cpu_baseline=rank == 0 and world_n == 1)
    except Exception as e:                                   # recorded, never fatal to the bench line
        line["remesh"] = {"error": str(e)[:300]}
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
