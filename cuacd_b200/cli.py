"""Command line: decompose mesh files into convex parts, one GLB per input
(the reference's `cuacd` command, cuacd/cli.py).

    python -m cuacd_b200 INPUT OUTPUT [options]

INPUT is a mesh file or a directory of them (.obj .stl .ply .off .glb
.gltf; -r also searches subdirectories).  OUTPUT receives <stem>.glb for
each input, under the input's directory relative to INPUT, with one node
per part named <stem>_<i> and one colour per part.  The options and their
defaults are the reference's (cuacd/cli.py:213-266).

Loading, decomposition and saving run as three spawned processes joined by
queues two items deep, so file work overlaps the GPU.  The decomposing
process owns the GPU context; when a mesh fails it closes the context, opens
a new one and tries that mesh once more.  A worker that dies without a
Python traceback (a native crash) ends the run: the supervisor stops the
other two and names the mesh the decomposer was working on.  --serial runs
the three steps in this process, one mesh at a time; --bench does the same
with a fresh context per mesh, an untimed first run (which sets the pool's
high-water mark) and a timed second run.

Before the search a mesh is remeshed (Context.preprocess at
--preprocess-resolution) when --preprocess is `on`, or, with the default
`auto`, when the GPU audit flags it (open, non-manifold or misoriented),
as the reference does (cuacd/cli.py:50-55).
"""
import argparse
import multiprocessing
import pathlib
import re
import sys
import time

import numpy as np

from . import meshio

_CUR_BYTES = 1024          # shared buffer holding the decomposer's current mesh name


def parse_pool_bytes(text):
    """Pool size with an optional K / M / G suffix (powers of 1,024); 0 = grow
    on demand (cuacd/cli.py:15-23)."""
    m = re.fullmatch(r"\s*(\d+(?:\.\d+)?)\s*([KMGkmg])?\s*", text)
    if not m:
        raise argparse.ArgumentTypeError(f"invalid pool size {text!r} (e.g. 512M, 2G, or 0 for on demand)")
    return int(float(m.group(1)) * {"": 1, "K": 1 << 10, "M": 1 << 20, "G": 1 << 30}[(m.group(2) or "").upper()])


def find_meshes(input_path, recursive):
    """[(absolute path, path relative to INPUT)] of the mesh files, sorted."""
    p = pathlib.Path(input_path).resolve()
    if p.is_file():
        return [(p, pathlib.Path(p.name))]
    if not p.is_dir():
        return []
    found = p.rglob("*") if recursive else p.iterdir()
    files = sorted(f for f in found if f.is_file() and f.suffix.lower() in meshio.MESH_EXTS)
    return [(f, f.relative_to(p)) for f in files]


def build_parser():
    ap = argparse.ArgumentParser(prog="cuacd_b200", description="GPU lookahead convex decomposition of mesh files.")
    ap.add_argument("input", help="mesh file or directory")
    ap.add_argument("output", help="output directory")
    ap.add_argument("-r", "--recursive", action="store_true", help="search subdirectories too")
    ap.add_argument("--width", type=int, default=30, help="candidate cuts per expansion level (30)")
    ap.add_argument("--width2", type=int, default=5, help="cuts at deeper expansion levels (5)")
    ap.add_argument("--depth", type=int, default=2, help="full expansion depth (2)")
    ap.add_argument("--quick-depth", type=int, default=0, help="quick expansion depth (0)")
    ap.add_argument("--threshold", type=float, default=0.05, help="convergence threshold (0.05)")
    ap.add_argument("--max-iters", type=int, default=100, help="outer iterations at most (100)")
    ap.add_argument("--device", type=int, default=-1, help="GPU ordinal; -1 keeps the current device")
    ap.add_argument("--pool", type=parse_pool_bytes, default=0, help="device pool size (K/M/G suffix; 0 = on demand)")
    ap.add_argument("--verbose", type=int, default=0, help="verbosity (0/1/2)")
    ap.add_argument("--debug", type=int, default=0, help="debug level (0/1)")
    ap.add_argument("--parts", action="store_true", help="save the cut parts instead of their convex hulls")
    ap.add_argument("--no-decompose-components", action="store_true",
                    help="do not split the input into connected components first")
    ap.add_argument("--no-decompose-components-per-iter", action="store_true",
                    help="do not split parts into connected components after each iteration")
    ap.add_argument("--n-concave-edges", type=int, default=16, help="concave edges sampled per cutting part (16)")
    ap.add_argument("--concave-eps", type=float, default=0.005, help="offset of edge-based planes (0.005)")
    ap.add_argument("--concave-threshold", type=float, default=3.49,
                    help="dihedral angle in radians above which an edge is concave (3.49)")
    ap.add_argument("--concave-iters", type=int, default=10, help="first iterations that sample concave edges (10)")
    ap.add_argument("--no-merge-hulls", dest="merge_hulls", action="store_false",
                    help="skip the greedy merge-hulls pass")
    ap.add_argument("--serial", action="store_true", help="load, decompose and save in this process")
    ap.add_argument("--preprocess", choices=["auto", "on", "off"], default="auto",
                    help="remesh to a watertight manifold first: auto (when the audit flags the mesh), on, off")
    ap.add_argument("--preprocess-resolution", type=int, default=64,
                    help="remesh grid resolution, a power of two (64)")
    ap.add_argument("--bench", action="store_true",
                    help="per mesh: fresh context, untimed run, timed run, pool high-water mark")
    return ap


def decompose_mesh(ctx, verts, tris, opts):
    """Parts of one mesh in its own coordinates: [(verts, tris)] of the
    parts' convex hulls (or, with opts.parts, of the cut parts).  The mesh
    is centred on its bounding box and scaled by half its longest side
    before the search and mapped back after (cuacd/cli.py:50-84)."""
    if opts.preprocess == "on" or (opts.preprocess == "auto" and ctx.check_mesh(verts, tris)["needs_remesh"]):
        verts, tris = ctx.preprocess(verts, tris, resolution=opts.preprocess_resolution)
    lo, hi = verts.min(axis=0), verts.max(axis=0)
    center = (lo + hi) / 2
    extent = float((hi - lo).max())
    scale = extent / 2 if extent > 0 else 1.0
    norm = ((verts - center) / scale).astype(np.float32)
    parts = ctx.lookahead_decompose(
        norm, tris, max_iters=opts.max_iters, width=opts.width, width2=opts.width2, depth=opts.depth,
        quick_depth=opts.quick_depth, threshold=opts.threshold, verbose=opts.verbose, debug=opts.debug,
        decompose_components=not opts.no_decompose_components,
        no_decompose_components_per_iter=opts.no_decompose_components_per_iter,
        n_concave_edges=opts.n_concave_edges, concave_eps=opts.concave_eps,
        concave_threshold=opts.concave_threshold, concave_iters=opts.concave_iters, merge_hulls=opts.merge_hulls)
    if opts.parts:
        return [(pv * scale + center, pt) for pv, pt, _, _ in parts]
    return [(hv * scale + center, ht) for _, _, hv, ht in parts]


def save_parts(parts, output_dir, rel_path):
    """Write <output_dir>/<rel_path's directory>/<stem>.glb; returns its path."""
    rel = pathlib.Path(rel_path)
    out_dir = pathlib.Path(output_dir) / rel.parent
    out_dir.mkdir(parents=True, exist_ok=True)
    out = out_dir / f"{rel.stem}.glb"
    data = meshio.glb_bytes(parts, [f"{rel.stem}_{i}" for i in range(len(parts))])
    tmp = out.with_suffix(".glb.part")
    tmp.write_bytes(data)
    tmp.replace(out)                     # a reader never sees half a file
    return out


def _default_context(device, pool_bytes):
    from . import Context
    return Context(device=device, pool_bytes=pool_bytes)


def _say(lock, msg, err=False):
    with lock:
        print(msg, file=sys.stderr if err else sys.stdout, flush=True)


# ---- pipeline workers (spawned processes) ---------------------------------
def _load_worker(items, q_out, lock):
    for abs_path, rel in items:
        try:
            v, t = meshio.load_mesh(abs_path)
        except Exception as e:                                  # a bad file is skipped
            _say(lock, f"{rel}: load error: {e}", err=True)
            continue
        q_out.put((str(rel), v, t))
    q_out.put(None)


def _decompose_worker(q_in, q_out, lock, opts, factory, current):
    ctx = factory(opts.device, opts.pool)
    try:
        while True:
            item = q_in.get()
            if item is None:
                break
            rel, v, t = item
            set_current(current, rel)
            t0 = time.perf_counter()
            parts = None
            for attempt in (0, 1):
                try:
                    parts = decompose_mesh(ctx, v, t, opts)
                    break
                except Exception as e:
                    if attempt:
                        _say(lock, f"{rel}: decompose error on retry: {e}", err=True)
                        break
                    _say(lock, f"{rel}: decompose error: {e}; reopening the context and retrying", err=True)
                    try:
                        ctx.close()
                    except Exception:
                        pass
                    ctx = factory(opts.device, opts.pool)
            if parts is not None:
                q_out.put((rel, parts, time.perf_counter() - t0))
    finally:
        ctx.close()
    q_out.put(None)


def _save_worker(q_in, output_dir, lock):
    while True:
        item = q_in.get()
        if item is None:
            break
        rel, parts, dt = item
        save_parts(parts, output_dir, rel)
        _say(lock, f"{rel}  {dt:.2f}s  {len(parts)} parts")


def supervise(workers, poll=0.05):
    """Wait for every (name, process) to end.  The first that exits with a
    non-zero code ends the others (they may be blocked on a queue it will
    never serve); returns its (name, exit code), or None when all end
    cleanly.  Each poll takes one liveness snapshot, so a worker that fails
    just as the last one ends is still seen."""
    while True:
        alive = [p.is_alive() for _, p in workers]
        for (name, p), up in zip(workers, alive):
            if not up and p.exitcode not in (0, None):
                for _, q in workers:
                    if q.is_alive():
                        q.terminate()
                for _, q in workers:
                    q.join()
                return name, p.exitcode
        if not any(alive):
            for _, p in workers:
                p.join()
            return None
        time.sleep(poll)


def set_current(buf, name):
    """Record in the shared buffer the mesh the decomposer is on (truncated
    to the buffer; a shorter name leaves no tail of the previous one)."""
    buf.value = str(name).encode("utf-8", "replace")[:_CUR_BYTES - 1]


def get_current(buf):
    return bytes(buf.value).decode("utf-8", "replace")


def run_pipeline(meshes, opts, factory):
    mp = multiprocessing.get_context("spawn")
    lock = mp.Lock()
    q_load, q_save = mp.Queue(maxsize=2), mp.Queue(maxsize=2)
    current = mp.Array("c", _CUR_BYTES)
    workers = [("loader", mp.Process(target=_load_worker, args=(meshes, q_load, lock))),
               ("decomposer", mp.Process(target=_decompose_worker,
                                         args=(q_load, q_save, lock, opts, factory, current))),
               ("saver", mp.Process(target=_save_worker, args=(q_save, opts.output, lock)))]
    for _, p in workers:
        p.start()
    failed = supervise(workers)
    if failed is None:
        return 0
    name, code = failed
    where = ""
    if name == "decomposer":
        mesh = get_current(current)
        if mesh:
            where = f" while decomposing {mesh!r}"
    cause = ("a native crash (killed by a signal, no traceback)" if code < 0
             else "an unhandled Python error (traceback above)")
    print(f"cuacd_b200: {name} exited with code {code}{where}: {cause}; stopping. "
          "Files written so far are complete.", file=sys.stderr, flush=True)
    return 1


def run_serial(meshes, opts, factory):
    for abs_path, rel in meshes:
        try:
            v, t = meshio.load_mesh(abs_path)
        except Exception as e:
            print(f"{rel}: load error: {e}", file=sys.stderr, flush=True)
            continue
        try:
            ctx = factory(opts.device, opts.pool)
        except Exception as e:
            print(f"{rel}: context error: {e}", file=sys.stderr, flush=True)
            continue
        try:
            if opts.bench:
                decompose_mesh(ctx, v, t, opts)                 # untimed: pool high-water mark
            t0 = time.perf_counter()
            parts = decompose_mesh(ctx, v, t, opts)
            dt = time.perf_counter() - t0
        except Exception as e:
            print(f"{rel}: decompose error: {e}", file=sys.stderr, flush=True)
            continue
        else:
            save_parts(parts, opts.output, rel)
            extra = f"  {ctx.pool_usage() / (1 << 20):.1f} MiB" if opts.bench else ""
            print(f"{rel}  {dt:.2f}s  {len(parts)} parts{extra}", flush=True)
        finally:
            ctx.close()
    return 0


def main(argv=None, context_factory=None):
    """Run the command; returns the exit code.  `context_factory(device,
    pool_bytes)` opens the GPU context (default: cuacd_b200.Context); for
    the pipelined mode it must be picklable (a module-level function)."""
    opts = build_parser().parse_args(argv)
    factory = context_factory or _default_context
    meshes = find_meshes(opts.input, opts.recursive)
    if not meshes:
        print(f"no mesh files found in {opts.input}", file=sys.stderr)
        return 1
    if opts.serial or opts.bench:
        return run_serial(meshes, opts, factory)
    return run_pipeline(meshes, opts, factory)


if __name__ == "__main__":
    sys.exit(main())
