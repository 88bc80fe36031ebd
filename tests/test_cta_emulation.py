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

from conftest import GOLDEN, ROOT, box_mesh
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
