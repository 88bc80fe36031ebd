"""Remesh front end (Context.preprocess) on the CPU.

- the library's marching-cubes table (cuacd_remesh_case_table, host code)
  is the oracle's, and contouring random fields with it gives closed,
  consistently oriented surfaces whose every vertex has one fan;
- the oracle (oracle/remesh.py) meets what the reference's own tests check
  (tests/test_preprocess.py there): an open cube, a doubled slab and a
  single triangle come out watertight and manifold, reversed winding gives
  the same shape, the extent grows by 2 (0.9 / R) margin, volume scales
  with the cube of the size and ignores translation, bad resolutions are
  refused;
- the remesh's device code, built for the host (tests/cta_emu/
  emu_remesh.cpp runs the per-item functions of remesh.cuh in the kernels'
  order), gives the oracle's vertices and triangles exactly."""
import collections
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, box_mesh
from cuacd_b200 import workloads as W
from oracle import remesh as RM

EMU = os.path.join(ROOT, "tests", "cta_emu")


def closed_manifold(t):
    """Every directed edge once with its reverse once, and the triangles
    around every vertex form one cycle."""
    e = collections.Counter()
    for a, b, c in np.asarray(t).tolist():
        for x, y in ((a, b), (b, c), (c, a)):
            e[(x, y)] += 1
    if not all(n == 1 and e.get((y, x), 0) == 1 for (x, y), n in e.items()):
        return False
    around = collections.defaultdict(dict)
    for a, b, c in np.asarray(t).tolist():
        for x, y, z in ((a, b, c), (b, c, a), (c, a, b)):
            if y in around[x]:
                return False
            around[x][y] = z
    for nxt in around.values():
        start = next(iter(nxt))
        cur, steps = nxt[start], 1
        while cur != start:
            cur = nxt.get(cur)
            steps += 1
            if cur is None or steps > len(nxt):
                return False
        if steps != len(nxt):
            return False
    return True


def volume(v, t):
    v = np.asarray(v, np.float64)
    return float(np.einsum("ij,ij->i", v[t[:, 0]], np.cross(v[t[:, 1]], v[t[:, 2]])).sum() / 6.0)


def no_zero_area(v, t):
    v = np.asarray(v, np.float32)
    cr = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
    return bool((np.abs(cr).sum(1) > 0).all())


def test_library_table_is_the_oracles():
    from cuacd_b200 import _fn
    out = (ctypes.c_int * (256 * 17))()
    _fn("cuacd_remesh_case_table")(ctypes.cast(out, ctypes.c_void_p))
    got = np.frombuffer(out, np.int32).reshape(256, 17)
    for case, loops in enumerate(RM.mc_case_table()):
        assert got[case, 0] == len(loops)
        assert got[case, 1:5].tolist() == [len(p) for p in loops] + [0] * (4 - len(loops))
        flat = [e for p in loops for e in p]
        assert got[case, 5:].tolist() == flat + [-1] * (12 - len(flat))


def test_table_contours_random_fields_closed():
    table = RM.mc_case_table()
    assert table[1] == [[0, 4, 8]] and table[254] == [[0, 8, 4]]    # corner 0 cut off, normal away from it
    rng = np.random.default_rng(0)
    for _ in range(150):
        R = int(rng.integers(3, 7))
        sd = rng.standard_normal((R, R, R)).astype(np.float32)
        sd[0], sd[-1], sd[:, 0], sd[:, -1], sd[:, :, 0], sd[:, :, -1] = 1, 1, 1, 1, 1, 1
        v, t = RM.contour(sd, R, table)
        if len(t):
            assert closed_manifold(t) and volume(v, t) > 0


@pytest.fixture(scope="module")
def cube():
    return box_mesh([0, 0, 0], [1, 1, 1])


def test_open_cube_doubled_slab_and_flat_triangle_heal(cube):
    v, t = cube
    for vv, tt in ((v, t[:10]),
                   (np.vstack([v, v + np.float32([0, 0, 1e-4])]), np.vstack([t, t[:, ::-1] + 8])),
                   (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]]))):
        rv, rt = RM.remesh(vv, tt, 16)
        assert len(rt) and closed_manifold(rt) and no_zero_area(rv, rt) and volume(rv, rt) > 0


def test_reversed_winding_same_shape(cube):
    v, t = cube
    a, b = RM.remesh(v, t, 16), RM.remesh(v, t[:, ::-1].copy(), 16)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("R", [16, 32])
def test_extent_grows_by_the_shift(cube, R):
    v, t = cube
    rv, rt = RM.remesh(v, t, R)
    margin = 1.0 + 2.0 * 3.0 / R
    assert float(rv[:, 0].max() - rv[:, 0].min()) == pytest.approx(1.0 + 2.0 * (0.9 / R) * margin, rel=0.02)


def test_scale_and_translation(cube):
    v, t = cube
    small = volume(*RM.remesh(v, t, 16))
    big = volume(*RM.remesh(v * 5 + np.float32([7, -3, 2]), t, 16))
    assert big / small == pytest.approx(125.0, rel=1e-3)


def test_bad_resolution(cube):
    for r in (48, 4, 0):
        with pytest.raises(ValueError):
            RM.remesh(*cube, r)


@pytest.fixture(scope="module")
def emu_remesh(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("emurm") / "emu_remesh")
    r = subprocess.run(["g++", "-std=c++20", "-O2", "-ffp-contract=off", os.path.join(EMU, "emu_remesh.cpp"),
                        "-o", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return out


def run_emu(exe, tmp_path, v, t, R):
    path = tmp_path / "in.bin"
    with open(path, "wb") as f:
        np.array([R, len(v), len(t)], np.int32).tofile(f)
        np.ascontiguousarray(v, np.float32).tofile(f)
        np.ascontiguousarray(t, np.int32).tofile(f)
    out = subprocess.run([exe, str(path)], capture_output=True, check=True, timeout=600).stdout
    nv, nt = np.frombuffer(out, np.int32, 2)
    ov = np.frombuffer(out, np.float32, 3 * nv, 8).reshape(-1, 3)
    ot = np.frombuffer(out, np.int32, 3 * nt, 8 + 12 * int(nv)).reshape(-1, 3)
    return ov, ot


def test_device_code_matches_the_oracle(emu_remesh, tmp_path, cube):
    v, t = cube
    sv, st = W.candidate_mesh(16, 8, 0.3, seed=1)
    for vv, tt, R in ((v, t, 16), (v, t[:10], 16), (sv, st, 32),
                      (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]]), 8)):
        ov, ot = RM.remesh(vv, tt, R)
        ev, et = run_emu(emu_remesh, tmp_path, vv, tt, R)
        np.testing.assert_array_equal(ev, ov)
        np.testing.assert_array_equal(et, ot)
