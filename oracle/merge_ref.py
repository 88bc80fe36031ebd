"""CPU restatement of the merge-hulls post-pass, for the tests.

TEST INFRASTRUCTURE ONLY (imported by tests/, never by the product).

Given the parts a search returned before merging, it decides which pairs the
post-pass merges, following the reference's pass (cuda/postprocess_merge.cu:
la_merge_cost_matrix :41-204, la_merge_hausdorff :205-405, la_merge_match
:406-492; csrc/lookahead.c:987-1063) with this library's deterministic
choices:

- candidate pairs (p1 > p2, in pair-index order) survive two quick rejects:
  the sum of the two hull-minus-mesh gaps already costing tau (FP32 rv
  formula, la_common.cuh:30-34), and boxes at least tau / 2 apart;
- the merged hull is the exact hull of both hulls' vertices (the oracle's
  hull, the same algorithm as the library's); its FP32 rv cost against the
  summed mesh volumes;
- below tau, the Hausdorff distance between the merged hull and both meshes
  concatenated less the triangles lying within 1e-3 of a shared plane -- the
  lowest face of the first part's hull with every vertex of that hull on or
  below it and every vertex of the second part's hull on it (merge.cuh);
  with no triangle left the distance is 0; cost = max(rv, Hausdorff);
- greedy matching: cheapest pair below tau first (ties: lower pair index),
  each part at most once.

A part's volumes are those the search carries: the hull volume of its hull
mesh, the mesh volume clamped to the hull volume (la_lifecycle.cu:294-297).
"""
import numpy as np

PI_F = np.float32(3.14159265358979)


def _rv_f32(gap):
    return np.float32(0.3) * np.cbrt(np.float32(3.0) / (np.float32(4.0) * PI_F) * np.float32(gap), dtype=np.float32)


def _vol64(v, t):
    v = np.asarray(v, np.float64)
    t = np.asarray(t)
    if len(t) == 0:
        return 0.0
    return abs(float(np.einsum("ij,ij->i", v[t[:, 0]], np.cross(v[t[:, 1]], v[t[:, 2]])).sum()) / 6.0)


def _shared_plane_filter(a, b, tol=np.float32(1e-3)):
    """Triangles of a then b (b's indices offset) less those within tol of
    the shared plane, as the library's merge kernel forms it (FP32)."""
    av, at, ahv, aht = a
    bv, bt, bhv, _ = b
    ahv32 = np.asarray(ahv, np.float32)
    bhv32 = np.asarray(bhv, np.float32)
    plane = None
    for f in range(len(aht)):
        ia, ib, ic = aht[f]
        A = ahv32[ia]
        e1, e2 = ahv32[ib] - A, ahv32[ic] - A
        n = np.cross(e1, e2).astype(np.float32)
        ln = np.float32(np.sqrt(np.float32(n @ n)))
        if ln < np.float32(1e-20):
            continue
        n = (n * (np.float32(1.0) / ln)).astype(np.float32)
        d = np.float32(n @ A)
        if (ahv32 @ n - d <= tol).all() and (np.abs(bhv32 @ n - d) <= tol).all():
            plane = (n, d)
            break
    tris = np.concatenate([np.asarray(at, np.int32), np.asarray(bt, np.int32) + len(av)])
    verts = np.concatenate([np.asarray(av, np.float32), np.asarray(bv, np.float32)])
    if plane is not None:
        n, d = plane
        s = np.abs(verts @ n - d) <= tol
        keep = ~(s[tris[:, 0]] & s[tris[:, 1]] & s[tris[:, 2]])
        tris = tris[keep]
    return verts, tris


def merge_pass(parts, tau, oracle):
    """parts: [(verts, tris, hull_verts, hull_tris)].  Returns (matches,
    costs): matches = [(p1, p2)] in the order they merge, costs = {(p1, p2):
    cost} of every candidate that reached the cost stage."""
    P = len(parts)
    tau = np.float32(tau)
    hvol = [_vol64(p[2], p[3]) for p in parts]
    mvol = [min(_vol64(p[0], p[1]), h) for p, h in zip(parts, hvol)]
    box = [(np.asarray(p[0], np.float32).min(0), np.asarray(p[0], np.float32).max(0)) for p in parts]
    cand = []
    for p1 in range(1, P):
        for p2 in range(p1):
            msum = np.float32(mvol[p1]) + np.float32(mvol[p2])
            gap = max(np.float32(np.float32(hvol[p1]) + np.float32(hvol[p2]) - msum), np.float32(0.0))
            if _rv_f32(gap) >= tau:
                continue
            (alo, ahi), (blo, bhi) = box[p1], box[p2]
            g = np.maximum(np.float32(0.0), np.maximum(alo - bhi, blo - ahi)).astype(np.float32)
            if np.float32(g @ g) >= (tau * np.float32(0.5)) ** 2:
                continue
            cand.append((p1, p2))
    costs = {}
    for p1, p2 in cand:
        A, B = parts[p1], parts[p2]
        pts = np.concatenate([np.asarray(A[2], np.float32), np.asarray(B[2], np.float32)])
        vidx, tris, hv = oracle.hull(pts)
        if len(tris) == 0:
            continue
        msum = np.float32(mvol[p1]) + np.float32(mvol[p2])
        rv = _rv_f32(max(np.float32(np.float32(hv) - msum), np.float32(0.0)))
        cost = float(rv)
        if rv < tau:
            mv, mt = _shared_plane_filter(A, B)
            if len(mt) > 0:
                h = oracle.hausdorff(pts[vidx], tris, mv, mt, threads=8)
                cost = max(cost, h)
        costs[(p1, p2)] = cost
    order = sorted((k for k in costs if costs[k] < tau), key=lambda k: (costs[k], k[0] * (k[0] - 1) // 2 + k[1]))
    used = set()
    matches = []
    for p1, p2 in order:
        if p1 in used or p2 in used:
            continue
        used.update((p1, p2))
        matches.append((p1, p2))
    return matches, costs
