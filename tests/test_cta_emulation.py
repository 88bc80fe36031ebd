"""Race detection on the CPU: the plane cut's device code (cut_cta) compiled
for the host by the CTA emulator in tests/cta_emu/ -- one std::thread per CUDA
thread, every __syncthreads and warp intrinsic checking that all live threads
reached the same call site.  The cut must raise no such report and must
produce the oracle's topology.

tests/golden/cut_ear_race.npz holds a part (4,938 triangles, the half of a
ridged sphere) and two planes on which the CTA ear clipping once let thread 0
relink the polygon while lagging threads still walked it; the threads then
met different barriers, which the GPU reports as an illegal instruction."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, box_mesh, box_with_cavity, nested_tori
from cuacd_b200 import workloads as W

EMU = os.path.join(ROOT, "tests", "cta_emu")


@pytest.fixture(scope="module")
def emu_cut(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("emu") / "emu_cut")
    r = subprocess.run(["g++", "-std=c++20", "-O2", "-pthread", "-ffp-contract=off", "-I", EMU,
                        os.path.join(EMU, "emu_cut.cpp"), "-o", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return out


def run(emu_cut, tmp_path, v, t, planes):
    path = str(tmp_path / "case.bin")
    with open(path, "wb") as f:
        np.array([len(v), len(t), len(planes)], np.int32).tofile(f)
        np.ascontiguousarray(v, np.float32).tofile(f)
        np.ascontiguousarray(t, np.int32).tofile(f)
        np.ascontiguousarray(planes, np.float32).tofile(f)
    r = subprocess.run([emu_cut, path], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    reports = [l for l in r.stderr.splitlines() if l.startswith("[emu]")]
    rows = []
    for line in r.stdout.splitlines():
        f = line.split()
        vals = dict(zip(f[2::2], (int(x) for x in f[3::2])))
        rows.append(vals)
    return rows, reports


def check(oracle, v, t, planes, rows):
    assert len(rows) == len(planes)
    for p, r in zip(planes, rows):
        pv, pt, nv_, nt_, info = oracle.plane_cut(v, t, p)
        assert r["err"] == 0
        assert (r["npv"], r["npt"], r["nnv"], r["nnt"]) == (len(pv), len(pt), len(nv_), len(nt_))
        assert r["cap"] == info["n_cap"] and r["loops"] == info["n_loops"]


def test_cube_and_sphere(emu_cut, tmp_path, oracle):
    v, t = box_mesh([0, 0, 0], [1, 1, 1])
    planes = np.array([[1, 0, 0, -0.5], [0.3, 0.4, 0.866, -0.9], [0, 0, 1, -1.0]], np.float32)
    rows, reports = run(emu_cut, tmp_path, v, t, planes)
    assert not reports, reports[:5]
    check(oracle, v, t, planes, rows)
    v, t = W.candidate_mesh(32, 12, 0.35, seed=3)
    planes = np.array([[1, 0, 0, 0.1], [0.6, 0.0, 0.8, -0.2], [0, 1, 0, 0.0]], np.float32)
    rows, reports = run(emu_cut, tmp_path, v, t, planes)
    assert not reports, reports[:5]
    check(oracle, v, t, planes, rows)


def test_ear_clipping_race_case(emu_cut, tmp_path, oracle):
    g = np.load(os.path.join(GOLDEN, "cut_ear_race.npz"))
    v, t, planes = g["v"], g["t"], g["planes"]
    rows, reports = run(emu_cut, tmp_path, v, t, planes)
    assert not reports, reports[:5]
    check(oracle, v, t, planes, rows)


def test_nested_loops_and_holes_emulated(emu_cut, tmp_path, oracle):
    """Caps with holes: loop nesting by ray crossings, and each hole bridged
    to its loop by CTA reductions (rightmost hole vertex, first edge met) and
    a parallel splice -- every barrier reached by the whole CTA, the
    oracle's loop and cap-triangle counts."""
    v, t = nested_tori()
    planes = []
    for plane in [(0, 0, 1, -0.013), (0.08, 0.05, 0.9955, -0.02), (1, 0, 0, -0.05)]:
        n = np.asarray(plane[:3], np.float64)
        planes.append([*(n / np.linalg.norm(n)), plane[3]])
    planes = np.asarray(planes, np.float32)
    rows, reports = run(emu_cut, tmp_path, v, t, planes)
    assert not reports, reports[:5]
    check(oracle, v, t, planes, rows)
    assert max(r["loops"] for r in rows) >= 6
    v, t = box_with_cavity()
    planes = np.array([[0, 0, 1, -0.5], [0.6, 0.48, 0.64, -0.9]], np.float32)
    rows, reports = run(emu_cut, tmp_path, v, t, planes)
    assert not reports, reports[:5]
    check(oracle, v, t, planes, rows)


def _cylinder(n, r=1.0, h=2.0):
    a = np.arange(n) * 2 * np.pi / n
    ring = np.stack([r * np.cos(a), r * np.sin(a), np.zeros(n)], 1)
    v = np.vstack([ring, ring + [0, 0, h], [[0, 0, 0], [0, 0, h]]]).astype(np.float32)
    t = []
    for i in range(n):
        j = (i + 1) % n
        t += [(i, j, n + j), (i, n + j, n + i), (2 * n, j, i), (2 * n + 1, n + i, n + j)]
    return v, np.asarray(t, np.int32)


def test_long_cap_and_touching_loops_emulated(emu_cut, tmp_path, oracle):
    """A 1,500-segment cylinder cut across: one 3,000-vertex cap, longer than
    the shared-memory ear buffers (ear clipping from global memory; loops
    traced by pointer jumping).  Two boxes that share an edge once their
    equal corners are merged: a plane across the edge gives two loops that
    touch (a vertex with two outgoing boundary edges: the serial walk), and
    a plane through their shared face fails its cap (the mesh goes back
    unsplit on the positive side)."""
    from conftest import l_shape
    from cuacd_b200 import meshio
    v, t = _cylinder(1500)
    planes = np.array([[0, 0, 1, -1.0]], np.float32)
    rows, reports = run(emu_cut, tmp_path, v, t, planes)
    assert not reports, reports[:5]
    check(oracle, v, t, planes, rows)
    assert rows[0]["cap"] == 2998
    mv, mt = meshio.clean_mesh(*l_shape())
    planes = np.array([[0, 0, 1, -0.25], [0, 1, 0, -0.5], [1, 0, 0, -1.0]], np.float32)
    rows, reports = run(emu_cut, tmp_path, mv, mt, planes)
    assert not reports, reports[:5]
    check(oracle, mv, mt, planes, rows)
    assert [oracle.plane_cut(mv, mt, p)[4]["cap_failed"] for p in planes] == [0, 1, 1]


def _l_prism():
    """The L-shaped prism of the reference's boundary-traversal regression
    (tests/test_boundary_loops.py:10-20 there): one closed manifold with a
    reflex edge, its six-gon sides split into quads."""
    xy = np.array([[0, 0], [2, 0], [2, 1], [1, 1], [1, 3], [0, 3]], np.float64)
    v = np.concatenate([np.column_stack([xy, np.zeros(6)]), np.column_stack([xy, np.ones(6)])])
    top = np.array([[0, 1, 3], [1, 2, 3], [0, 3, 5], [3, 4, 5]])
    f = list(top[:, [0, 2, 1]]) + list(top + 6)
    for i in range(6):
        j = (i + 1) % 6
        f += [[i, j, j + 6], [i, j + 6, i + 6]]
    lo, hi = v.min(0), v.max(0)
    v = (v - (lo + hi) / 2) / ((hi - lo).max() / 2)
    return v.astype(np.float32), np.asarray(f, np.int32)


def test_l_prism_cuts_emulated(emu_cut, tmp_path, oracle):
    """Planes through the L-prism's notch, along its faces and oblique:
    every barrier reached by the whole CTA, the oracle's counts."""
    v, t = _l_prism()
    planes = np.array([[1, 0, 0, 0.0], [0, 1, 0, 0.3333333], [0, 0, 1, 0.0], [1, 0, 0, 0.3333333],
                       [0.6, 0.8, 0, -0.1], [0.48, 0.36, 0.8, 0.05], [0, 1, 0, -0.3333333]], np.float32)
    rows, reports = run(emu_cut, tmp_path, v, t, planes)
    assert not reports, reports[:5]
    check(oracle, v, t, planes, rows)


def _build_emu_hull(tmp_path_factory, defines=()):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("emuh") / "emu_hull")
    r = subprocess.run(["g++", "-std=c++20", "-O2", "-pthread", "-ffp-contract=off", *defines, "-I", EMU,
                        os.path.join(EMU, "emu_hull.cpp"), "-o", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return out


@pytest.fixture(scope="module")
def emu_hull(tmp_path_factory):
    return _build_emu_hull(tmp_path_factory)


@pytest.fixture(scope="module")
def emu_hull_small_lists(tmp_path_factory):
    """The same pipeline with 64 shared ints per warp (a 40-node stack and a
    24-leaf list) instead of 1,024, so that wraps hit the stack limiter,
    the leaf-list compaction and the fall-back to the hull's own lists."""
    return _build_emu_hull(tmp_path_factory, ["-DHULL_WSM=64", "-DHULL_WQ=40"])


def run_hulls(emu_hull, tmp_path, clouds):
    path = str(tmp_path / "clouds.bin")
    with open(path, "wb") as f:
        np.array([len(clouds)] + [len(c) for c in clouds], np.int32).tofile(f)
        for c in clouds:
            np.ascontiguousarray(c, np.float32).tofile(f)
    r = subprocess.run([emu_hull, path], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    reports = [l for l in r.stderr.splitlines() if l.startswith("[emu]")]
    lines = r.stdout.splitlines()
    out = []
    for i in range(0, len(lines), 3):
        h = lines[i].split()
        err, nv, nt = int(h[3]), int(h[5]), int(h[7])
        v = np.array(lines[i + 1].split(), np.float32).reshape(nv, 3)
        t = np.array(lines[i + 2].split(), np.int32).reshape(nt, 3)
        out.append((err, v, t))
    return out, reports


def test_hull_pipeline_emulated(emu_hull, tmp_path, oracle):
    """The batched hull pipeline's set-up, wrap and output code (one wrap CTA
    for every cloud) raises no divergent barrier or warp misuse and builds
    the oracle's hulls: uniform clouds, a fragment of a cut (a large flat cap
    face), flat leaves lying in faces, duplicated points, a grid with many
    coplanar points, and clouds with 34 points on their lexicographic minimum
    (a collinear first contact set)."""
    rng = np.random.default_rng(4)
    v, t = W.candidate_mesh(32, 12, 0.35, seed=3)
    frag = oracle.plane_cut(v, t, np.array([0.6, 0.0, 0.8, -0.2], np.float32))[0]
    dup = rng.uniform(-1, 1, (200, 3)).astype(np.float32)
    dup = np.concatenate([dup, dup[:40]])
    g = np.stack(np.meshgrid(*[np.linspace(-1, 1, 6)] * 3), -1).reshape(-1, 3).astype(np.float32)
    dc = np.load(os.path.join(GOLDEN, "hull_dup_corner.npz"))
    clouds = W.hull_clouds(3, 600, 0) + [frag, np.load(os.path.join(GOLDEN, "hull_flat_leaves.npy")), dup, g,
                                         dc["c0"], dc["c1"]]
    got, reports = run_hulls(emu_hull, tmp_path, clouds)
    assert not reports, reports[:5]
    for c, (err, hv, ht) in zip(clouds, got):
        vi, tri, vol = oracle.hull(c)
        assert err == 0
        np.testing.assert_array_equal(hv, c[vi])
        np.testing.assert_array_equal(ht, tri)


def test_hull_overflow_paths_emulated(emu_hull_small_lists, tmp_path, oracle):
    """With small per-warp lists, sphere shells and uniform clouds (many
    leaves kept near each wrapping plane) still give the oracle's hulls, with
    no divergent barrier or warp misuse, through the stack limiter, the
    compaction of the kept-leaf list and the hull's own (locked) lists."""
    rng = np.random.default_rng(5)
    shells = []
    for n in (1500, 3000):
        d = rng.normal(size=(n, 3))
        shells.append((d / np.linalg.norm(d, axis=1, keepdims=True) * rng.uniform(0.98, 1.0, (n, 1))).astype(np.float32))
    clouds = shells + W.hull_clouds(2, 2000, 6)
    got, reports = run_hulls(emu_hull_small_lists, tmp_path, clouds)
    assert not reports, reports[:5]
    for c, (err, hv, ht) in zip(clouds, got):
        vi, tri, vol = oracle.hull(c)
        assert err == 0
        np.testing.assert_array_equal(hv, c[vi])
        np.testing.assert_array_equal(ht, tri)


@pytest.fixture(scope="module", params=[8, 32])
def emu_hull_leaf(request, tmp_path_factory):
    """The pipeline built with BVH leaves of 8 or 32 points instead of 16."""
    return _build_emu_hull(tmp_path_factory, [f"-DHULL_LEAF={request.param}"])


def test_hull_leaf_sizes_emulated(emu_hull_leaf, tmp_path, oracle):
    """Every kernel of the hull pipeline takes its leaf size from HULL_LEAF
    (the seed scan included): with leaves of 8 and of 32 points the hulls
    are still the oracle's, with no divergent barrier or warp misuse."""
    v, t = W.candidate_mesh(32, 12, 0.35, seed=3)
    frag = oracle.plane_cut(v, t, np.array([0.6, 0.0, 0.8, -0.2], np.float32))[0]
    rng = np.random.default_rng(9)
    d = rng.normal(size=(1500, 3))
    shell = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    clouds = W.hull_clouds(2, 700, 1) + [frag, shell, np.load(os.path.join(GOLDEN, "hull_flat_leaves.npy"))]
    got, reports = run_hulls(emu_hull_leaf, tmp_path, clouds)
    assert not reports, reports[:5]
    for c, (err, hv, ht) in zip(clouds, got):
        vi, tri, vol = oracle.hull(c)
        assert err == 0
        np.testing.assert_array_equal(hv, c[vi])
        np.testing.assert_array_equal(ht, tri)


@pytest.fixture(scope="module")
def emu_hd(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("emuhd") / "emu_hd")
    r = subprocess.run(["g++", "-std=c++20", "-O2", "-pthread", "-ffp-contract=off", "-I", EMU,
                        os.path.join(EMU, "emu_hd.cpp"), "-o", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return out


def test_hausdorff_query_emulated(emu_hd, tmp_path, oracle):
    """The Hausdorff prep and query (cuacd_b200/csrc/hausdorff.cuh) run
    on the CPU: every barrier and warp vote is reached by the whole CTA /
    warp from one site (the query's warps vote inside loops whose lanes
    search different BVH paths; a lane that skipped a vote would hang the
    warp on the GPU), and the distance equals the oracle's within 1e-5.
    Cases: a sphere against its hull, nested boxes, and a tetrahedron
    (a one-leaf BVH) against an icosphere, both directions each."""
    from cuacd_b200 import workloads as W
    v, t = W.hausdorff_sphere(level=3)
    hvi, htri, _ = oracle.hull(v)
    tet = (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32),
           np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.int32))
    cases = [((v[hvi], htri), (v, t)), (box_mesh([-1] * 3, [1] * 3), box_mesh([-.5] * 3, [.5] * 3)),
             (tet, W.icosphere(1))]
    for k, (a, b) in enumerate(cases):
        path = str(tmp_path / f"hd{k}.bin")
        with open(path, "wb") as f:
            np.array([len(a[0]), len(a[1]), len(b[0]), len(b[1]), 1000, 0], np.int32).tofile(f)
            np.array([2000.0], np.float32).tofile(f)
            for x in (a[0], a[1], b[0], b[1]):
                np.ascontiguousarray(x, np.float32 if x.dtype.kind == "f" else np.int32).tofile(f)
        r = subprocess.run([emu_hd, path], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0 and "[emu]" not in r.stderr, r.stderr[-2000:]
        d = float(r.stdout.split()[0])
        o = oracle.hausdorff(a[0], a[1], b[0], b[1], threads=8)
        assert abs(d - o) < 1e-5, (k, d, o)
