"""Generate the golden fixtures in tests/golden/ (run in a checkout that has
the reference tree and scipy; the fixtures are committed, so tests never
need either).

  hull_qhull.npz      point clouds; their hull-grid coordinates computed by an
                      independent numpy float32 restatement of the quantiser
                      (cuda/hull_dandc.cuh:1366-1408); scipy/Qhull vertex sets
                      on those grid points; Qhull volumes of the float points.
  hausdorff_ref.npz   the reference's golden Hausdorff pairs and CoACD values
                      (tests/data/hausdorff_coacd_ref.npz in the reference).

usage: python tests/golden/make_golden.py path/to/reference
"""
import os
import sys

import numpy as np
import scipy.spatial

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from cuacd_b200 import workloads as W  # noqa: E402


def quantize_np(pts):
    """float32 restatement of the hull grid (numpy: IEEE ops, no FMA)."""
    p = np.asarray(pts, np.float32)
    mn, mx = p.min(0), p.max(0)
    span = (mx - mn).astype(np.float32)
    s0, s1, s2 = span
    max_ax = (0 if s0 >= s2 else 2) if s0 >= s1 else (1 if s1 >= s2 else 2)
    min_ax = (0 if s0 <= s2 else 2) if s0 <= s1 else (1 if s1 <= s2 else 2)
    if min_ax == max_ax:
        min_ax = (max_ax + 1) % 3
    med_ax = 3 - max_ax - min_ax
    sc = (span / np.float32(10216.0)).astype(np.float32)
    if (med_ax + 1) % 3 != max_ax:
        sc = -sc
    cen = ((mn + mx) * np.float32(0.5)).astype(np.float32)
    q = np.empty((len(p), 3), np.int32)
    for k, a in enumerate((med_ax, max_ax, min_ax)):
        inv = np.float32(1.0) / sc[a] if sc[a] != 0 else np.float32(0.0)
        d = (p[:, a] - cen[a]).astype(np.float32)
        q[:, k] = np.trunc((d * np.float32(inv)).astype(np.float32)).astype(np.int32)
    return q


def clouds():
    out = []
    names = []
    for i, c in enumerate(W.hull_clouds(12, 1000, 0)):
        out.append(c); names.append(f"cube_uniform_{i}")
    rng = np.random.default_rng(11)
    for n in (20, 200, 2000):
        g = rng.standard_normal((n, 3)).astype(np.float32)
        out.append(g); names.append(f"gaussian_{n}")
        s = rng.standard_normal((n, 3))
        s /= np.linalg.norm(s, axis=1, keepdims=True)
        out.append(s.astype(np.float32)); names.append(f"sphere_shell_{n}")
    v, _ = W.hausdorff_sphere(level=3)
    out.append(v); names.append("displaced_icosphere_l3")
    return out, names


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <path of the reference tree>")
    ref = sys.argv[1]
    cl, names = clouds()
    rec = {"names": np.array(names)}
    for i, c in enumerate(cl):
        q = quantize_np(c)
        qh = scipy.spatial.ConvexHull(q.astype(np.float64))
        fh = scipy.spatial.ConvexHull(c.astype(np.float64))
        rec[f"pts_{i}"] = c
        rec[f"q_{i}"] = q
        rec[f"qhull_vertices_{i}"] = np.sort(qh.vertices).astype(np.int32)
        rec[f"qhull_volume_{i}"] = np.float64(fh.volume)
    rec["n"] = np.int64(len(cl))
    np.savez_compressed(os.path.join(HERE, "hull_qhull.npz"), **rec)

    src = os.path.join(ref, "tests", "data", "hausdorff_coacd_ref.npz")
    d = np.load(src, allow_pickle=True)
    hd = {"n_pairs": np.int64(d["n_pairs"]), "names": np.array([str(x) for x in d["names"]])}
    for i in range(int(d["n_pairs"])):
        for k in ("verts_a", "verts_b"):
            hd[f"{k}_{i}"] = d[f"{k}_{i}"].astype(np.float32)
        for k in ("tris_a", "tris_b"):
            hd[f"{k}_{i}"] = d[f"{k}_{i}"].astype(np.int32)
        hd[f"ref_{i}"] = np.float64(d[f"ref_{i}"])
    np.savez_compressed(os.path.join(HERE, "hausdorff_ref.npz"), **hd)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
