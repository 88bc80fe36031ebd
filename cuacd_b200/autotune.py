"""Autotuner of the batched hull pipeline's launch shape.

The hull pipeline (hull.cu) has two launch-shape choices that the best
value of depends on the batch and the device:

- points per wrap CTA: how many of the batch's points one persistent wrap
  CTA (16 warps) stands for, i.e. how many warps share a cloud; the grid is
  the batch's points / this, at most the resident CTAs of the device;
- the seed threshold: clouds of at least this many points start wrapping
  from six seed faces (extreme points along +-x, +-y, +-z) instead of one,
  which widens the frontier of a large cloud from the start but costs set-up
  time on a small one.

They are tuned per size class of a batch's largest cloud (0: < 4,096
points, 1: < 65,536, 2: larger) on representative batches of that class:
the config-1 clouds (256 x 1,000 uniform points); the fragments that the 30
candidate planes cut from the config-3 sphere (5,000-20,000 points each)
and, alone, the vertices of a 81,920-triangle displaced sphere of config 4
(40,962 points, the input hull a lookahead search starts from); and two
163,842-point clouds (a level-7 icosphere, all of whose points are on its
hull, and the largest displaced sphere of config 4).  Each shape is timed
with CUDA events on device-resident inputs (median of `reps` calls after a
warm-up call, summed over the class's batches); the fastest is applied
through
cuacd_hull_set_tuning and, with --write, stored per device name in
tuning.json beside this file, which Context applies when it opens a device
of that name.  The results are the same for every shape (the hull output
is canonical); only the time changes.

usage:  python -m cuacd_b200.autotune [--write] [--reps N]
"""
import ctypes
import json
import os
import statistics
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TUNING_PATH = os.path.join(HERE, "tuning.json")
CLASSES = (0, 1, 2)
PTS_PER_CTA = (1024, 2048, 4096, 8192, 16384)
SEED_MIN_N = {0: (0,), 1: (0, 4096), 2: (0, 65536)}


def device_name(ctx):
    from . import _fn
    buf = ctypes.create_string_buffer(256)
    n_sm = ctypes.c_int(0)
    ctx._check(_fn("cuacd_device_info")(ctx.handle, buf, 256, ctypes.byref(n_sm)))
    return buf.value.decode(), int(n_sm.value)


def set_tuning(ctx, cls, pts_per_cta, seed_min_n):
    from . import _fn
    ctx._check(_fn("cuacd_hull_set_tuning")(ctx.handle, int(cls), int(pts_per_cta), int(seed_min_n)))


def get_tuning(ctx, cls):
    from . import _fn
    a, b = ctypes.c_int(0), ctypes.c_int(0)
    ctx._check(_fn("cuacd_hull_get_tuning")(ctx.handle, int(cls), ctypes.byref(a), ctypes.byref(b)))
    return int(a.value), int(b.value)


def apply_stored(ctx, path=TUNING_PATH):
    """Apply the stored tuning of this device's name, if any; returns it."""
    try:
        with open(path) as f:
            table = json.load(f)
    except (OSError, ValueError):
        return None
    name, _ = device_name(ctx)
    entry = table.get(name)
    if not entry:
        return None
    for cls, (ppc, seed) in enumerate(entry.get("hull", [])):
        set_tuning(ctx, cls, ppc, seed)
    return entry


def workloads(ctx):
    """Representative batches of each size class (see the module
    docstring): {class: [batch, ...]}, a batch being a list of clouds."""
    from . import workloads as W
    out = {0: [W.hull_clouds(256, 1000, 0)]}
    v, t = W.candidate_mesh()
    conc, axis, valid = ctx.candidate_planes(v, t, 16, 0.005, 3.49, 3, 0.0125)
    planes = np.concatenate([conc[:27], axis[valid]]).astype(np.float32)
    frags = []
    for p in planes:
        pv, pt, nv, nt = ctx.plane_cut(v, t, p)
        if len(pt) and len(nt):
            frags += [pv, nv]
    sample = W.batch_meshes(512, 500, 200_000, seed=3, select={i for i in range(512) if i % 16 in (0, 5)})
    lone = next(m[0] for m in sample if len(m[1]) == 81920)
    out[1] = [frags, [lone]]
    iv, _ = W.icosphere(7)
    big = max(sample, key=lambda m: len(m[0]))
    out[2] = [[iv.astype(np.float32), big[0]]]
    return out


class _Batch:
    """Device-resident hull batch timed with CUDA events."""

    def __init__(self, ctx, clouds):
        import torch
        from . import _fn
        self.ctx, self.fn = ctx, _fn("cuacd_hull_batch_device")
        self.n = len(clouds)
        self.max_pts = max(len(c) for c in clouds)
        packed = np.ascontiguousarray(np.concatenate(clouds), np.float32)
        off = np.zeros(self.n + 1, np.int32)
        off[1:] = np.cumsum([len(c) for c in clouds])
        self.max_ht = max(2 * self.max_pts - 4, 4)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.pts = torch.from_numpy(packed.reshape(-1)).to(dev)
        self.off = torch.from_numpy(off).to(dev)
        self.v = torch.empty(self.n * self.max_pts * 3, dtype=torch.float32, device=dev)
        self.t = torch.empty(self.n * self.max_ht * 3, dtype=torch.int32, device=dev)
        self.nv, self.nt, self.err = (torch.empty(self.n, dtype=torch.int32, device=dev) for _ in range(3))
        self.vol = torch.empty(self.n, dtype=torch.float32, device=dev)
        self.stream = torch.cuda.Stream(device=dev)

    def run(self):
        P = lambda x: ctypes.c_void_p(x.data_ptr())
        self.ctx._check(self.fn(self.ctx.handle, P(self.pts), P(self.off), self.n, self.max_pts, self.max_pts,
                                self.max_ht, P(self.v), P(self.t), P(self.nv), P(self.nt), P(self.vol), P(self.err),
                                ctypes.c_void_p(self.stream.cuda_stream)))

    def time_ms(self, reps):
        import torch
        with torch.cuda.stream(self.stream):
            self.run()
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
            for a, b in ev:
                a.record(self.stream)
                self.run()
                b.record(self.stream)
            self.stream.synchronize()
        if int(self.err.abs().sum()):
            raise RuntimeError("hull errors during tuning")
        return statistics.median(a.elapsed_time(b) for a, b in ev)

    def result(self):
        return self.nv.cpu().numpy().copy(), self.nt.cpu().numpy().copy(), self.vol.cpu().numpy().copy()


def tune(ctx, reps=5, pts_per_cta=PTS_PER_CTA, seed_min_n=SEED_MIN_N, batches=None):
    """Sweep every size class; applies and returns {"hull": [[ppc, seed] per
    class], "ms": {class: {"ppc/seed": ms}}}."""
    batches = batches if batches is not None else workloads(ctx)
    table, times = [], {}
    for cls in CLASSES:
        group = batches[cls]
        if len(group) and isinstance(group[0], np.ndarray):     # one batch given as its clouds
            group = [group]
        bs = [_Batch(ctx, g) for g in group]
        times[cls] = {}
        best = None
        refs = [None] * len(bs)
        for ppc in pts_per_cta:
            for seed in seed_min_n[cls]:
                set_tuning(ctx, cls, ppc, seed)
                ms = 0.0
                for k, b in enumerate(bs):
                    ms += b.time_ms(reps)
                    res = b.result()
                    if refs[k] is None:
                        refs[k] = res
                    elif not all(np.array_equal(x, y) for x, y in zip(refs[k], res)):
                        raise RuntimeError(f"class {cls}: hull results changed with the launch shape {ppc}/{seed}")
                times[cls][f"{ppc}/{seed}"] = ms
                if best is None or ms < best[0]:
                    best = (ms, ppc, seed)
        set_tuning(ctx, cls, best[1], best[2])
        table.append([best[1], best[2]])
    return {"hull": table, "ms": times}


def main(argv):
    import cuacd_b200
    reps = int(argv[argv.index("--reps") + 1]) if "--reps" in argv else 5
    with cuacd_b200.Context(0) as ctx:
        name, n_sm = device_name(ctx)
        for cls in CLASSES:
            set_tuning(ctx, cls, 0, 0)
        res = tune(ctx, reps)
        print(json.dumps({"device": name, "n_sm": n_sm, **res}, indent=1))
        if "--write" in argv:
            try:
                with open(TUNING_PATH) as f:
                    table = json.load(f)
            except (OSError, ValueError):
                table = {}
            table[name] = {"hull": res["hull"], "n_sm": n_sm, "measured_ms": res["ms"],
                           "how": f"python -m cuacd_b200.autotune --reps {reps}: CUDA-event median per "
                                  "launch shape of each size class's batch"}
            with open(TUNING_PATH, "w") as f:
                json.dump(table, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:])
