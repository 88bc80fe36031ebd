"""CPU restatement of the remesh front end (Context.preprocess), for tests
only: the CUDA path in cuacd_b200/csrc/remesh.cu is checked against it
value for value.  Test infrastructure; nothing in the library imports it.

The pipeline follows the reference's stages and conventions
(csrc/preprocess.c:1-13, 605-700): the mesh is normalised into a padded
unit cube, p_norm = ((p - vmin) / extent + band) / margin with band = 3/R
and margin = 1 + 2 band, and grid node g samples p_norm = (g + 0.5) / R;
an unsigned distance field is computed within `band` (3 cells) of the
triangles, signed by a flood fill from the grid's boundary that no grid
edge crossed by a triangle lets through, shifted by 0.9/R (one node in
0.9 cells of the surface already counts as inside, so the surface grows by
0.9 cells), and contoured at 0; vertices map back by
p = ((g + 0.5) / R * margin - band) * extent + vmin.  The reference reaches
the same stages through a third-party rasteriser and a dual marching-cubes
port; the contouring here is marching cubes with a case table generated
from one rule (below), which makes every output closed, manifold and
consistently oriented.  Parity with the reference is on the properties its
own tests check (tests/test_preprocess.py); vertex positions: parity
unpinned (the reference's dual contouring places them differently).

Everything is in grid units (u = p_norm * R - 0.5, nodes at integers) and
float64 in a fixed operation order, which the CUDA path repeats (compiled
without FMA contraction):
  squared distance node-triangle: min of the three segment distances and,
    when the node projects inside, the plane distance;
  a node keeps float32(d2) when d2 <= 9 (band squared), the least over
    triangles; other nodes are far;
  a grid edge (node, node + e_k) is crossed when the line through the
    node's other two coordinates meets the triangle (inclusive 2D test in
    the projection) at a k-coordinate z with floor(z) = node_k;
  field = (outside ? u : -u) - 0.9 with u = sqrt(d2) (1e9 when far),
    rounded to float32; a node is inside when field < 0.
"""
import numpy as np

BAND_CELLS = 3.0
SHIFT_CELLS = 0.9
T_CLAMP = 0.01
FAR_D2 = np.float32(np.finfo(np.float32).max)

# cube corners c: (x, y, z) = (c & 1, c >> 1 & 1, c >> 2 & 1); edges axis by
# axis, each from the corner with that bit clear
EDGES = [(c, c | (1 << a), a) for a in range(3) for c in range(8) if not c >> a & 1]


def _edge_of(c0, c1):
    lo, hi = min(c0, c1), max(c0, c1)
    for e, (a, b, _) in enumerate(EDGES):
        if (a, b) == (lo, hi):
            return e
    raise ValueError("not a cube edge")


def _faces():
    """Each face's corners in counter-clockwise order seen from outside."""
    out = []
    for a in range(3):
        b, c = (a + 1) % 3, (a + 2) % 3
        for s in (0, 1):
            cyc = []
            for (pb, pc) in ((0, 0), (1, 0), (1, 1), (0, 1)):
                cyc.append((s << a) | (pb << b) | (pc << c))
            out.append(cyc if s else cyc[::-1])
    return out


def mc_case_table():
    """Marching-cubes loops of each of the 256 cases: a list of polygons,
    each a list of cube edges in the order whose right-hand normal points
    from inside to outside.

    On each face, a segment runs from every edge where the cycle goes from
    an inside corner to an outside one back to the edge that opened that
    run of inside corners; on a face with two diagonal inside corners each
    is cut off by its own segment (the inside is 6-connected), a rule that
    depends only on the face, so neighbouring cells agree.  Every crossed
    edge then starts one segment and ends one, and the segments close into
    loops, each reversed and started at its first edge.  A loop of three
    is one triangle; a longer one is fanned around a vertex at the mean of
    its points (a fan from a corner could join two points of one face, as
    the neighbouring cell may, and four triangles would share that
    edge)."""
    faces = _faces()
    table = []
    for case in range(256):
        inside = [bool(case >> c & 1) for c in range(8)]
        nxt = {}
        for cyc in faces:
            st = [inside[q] for q in cyc]
            for i in range(4):
                if st[i] and not st[(i + 1) % 4]:              # inside -> outside at edge i
                    j = i
                    while st[j]:                                # back to the run's first corner
                        j = (j - 1) % 4
                    nxt[_edge_of(cyc[i], cyc[(i + 1) % 4])] = _edge_of(cyc[j], cyc[(j + 1) % 4])
        seen, out = set(), []
        for e in range(12):
            if e not in nxt or e in seen:
                continue
            loop = [e]
            seen.add(e)
            f = nxt[e]
            while f != e:
                loop.append(f)
                seen.add(f)
                f = nxt[f]
            out.append([loop[0]] + loop[1:][::-1])
        table.append(out)
    return table


def normalise(verts, R):
    """(grid-unit vertices float64, vmin float32[3], extent float32,
    band, margin)."""
    v = np.asarray(verts, np.float32).reshape(-1, 3)
    vmin, vmax = v.min(0), v.max(0)
    extent = np.float32(max(vmax[d] - vmin[d] for d in range(3)))
    band = 3.0 / R
    margin = 1.0 + 2.0 * band
    u = ((v.astype(np.float64) - vmin.astype(np.float64)) / np.float64(extent) + band) / margin * R - 0.5
    return u, vmin, extent, band, margin


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], -1)


def _seg_d2(P, A, B):
    AB = B - A
    ll = _dot(AB, AB)
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.where(ll > 0, _dot(P - A, AB) / np.where(ll > 0, ll, 1.0), 0.0)
    t = np.minimum(np.maximum(t, 0.0), 1.0)
    D = P - (A + t[..., None] * AB)
    return _dot(D, D)


def point_tri_d2(P, A, B, C):
    """Squared distance of points P (..., 3) to triangles ABC (float64;
    A, B, C broadcast against P, one triangle per leading index)."""
    AB, BC, CA = B - A, C - B, A - C
    n = _cross(AB, C - A)
    nn = _dot(n, n)
    d2 = np.minimum(np.minimum(_seg_d2(P, A, B), _seg_d2(P, B, C)), _seg_d2(P, C, A))
    with np.errstate(divide="ignore", invalid="ignore"):
        s0 = _dot(_cross(AB, P - A), n)
        s1 = _dot(_cross(BC, P - B), n)
        s2 = _dot(_cross(CA, P - C), n)
        dp = _dot(P - A, n)
        inside = (nn > 0) & (s0 >= 0) & (s1 >= 0) & (s2 >= 0)
        return np.where(inside, np.minimum(d2, dp * dp / np.where(nn > 0, nn, 1.0)), d2)


def distance_grid(u, tris, R, chunk=2048):
    """float32 squared distance per node [z, y, x], FAR_D2 beyond the band.
    Triangles whose node boxes have the same shape are evaluated together;
    the least value per node does not depend on the order."""
    g = np.full(R * R * R, FAR_D2, np.float32)
    T = np.asarray(tris).reshape(-1, 3)
    A, B, C = u[T[:, 0]], u[T[:, 1]], u[T[:, 2]]
    lo = np.maximum(np.ceil(np.minimum(np.minimum(A, B), C) - BAND_CELLS), 0).astype(np.int64)
    hi = np.minimum(np.floor(np.maximum(np.maximum(A, B), C) + BAND_CELLS), R - 1).astype(np.int64)
    dims = hi - lo + 1
    keep = np.flatnonzero((dims > 0).all(1))
    shapes, group = np.unique(dims[keep], axis=0, return_inverse=True)
    for gi, (nx, ny, nz) in enumerate(shapes):
        members = keep[group.reshape(-1) == gi]
        zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        off = np.stack([xx, yy, zz], -1).reshape(-1, 3)                      # box nodes, x fastest
        for c0 in range(0, len(members), chunk):
            m = members[c0:c0 + chunk]
            node = lo[m][:, None, :] + off[None, :, :]                       # (tris, nodes, 3)
            d2 = point_tri_d2(node.astype(np.float64), A[m][:, None, :], B[m][:, None, :], C[m][:, None, :])
            sel = d2 <= BAND_CELLS * BAND_CELLS
            lin = (node[..., 2] * R + node[..., 1]) * R + node[..., 0]
            np.minimum.at(g, lin[sel], d2[sel].astype(np.float32))
    return g.reshape(R, R, R)


def _orient(X, Y, Pi, Pj, i, j):
    return (Y[i] - X[i]) * (Pj - X[j]) - (Y[j] - X[j]) * (Pi - X[i])


def crossed_edges(u, tris, R, chunk=4096):
    """bool [3][z, y, x]: grid edge from the node along axis k is crossed.
    Per axis, triangles whose line boxes have the same shape are tested
    together (the marks do not depend on the order)."""
    blk = np.zeros((3, R * R * R), bool)
    T = np.asarray(tris).reshape(-1, 3)
    A, B, C = u[T[:, 0]], u[T[:, 1]], u[T[:, 2]]
    for k in range(3):
        i, j = (k + 1) % 3, (k + 2) % 3
        area = (B[:, i] - A[:, i]) * (C[:, j] - A[:, j]) - (B[:, j] - A[:, j]) * (C[:, i] - A[:, i])
        a0 = np.maximum(np.ceil(np.minimum(np.minimum(A[:, i], B[:, i]), C[:, i])), 0).astype(np.int64)
        a1 = np.minimum(np.floor(np.maximum(np.maximum(A[:, i], B[:, i]), C[:, i])), R - 1).astype(np.int64)
        b0 = np.maximum(np.ceil(np.minimum(np.minimum(A[:, j], B[:, j]), C[:, j])), 0).astype(np.int64)
        b1 = np.minimum(np.floor(np.maximum(np.maximum(A[:, j], B[:, j]), C[:, j])), R - 1).astype(np.int64)
        dims = np.stack([a1 - a0 + 1, b1 - b0 + 1], 1)
        keep = np.flatnonzero((area != 0) & (dims > 0).all(1))
        if len(keep) == 0:
            continue
        shapes, group = np.unique(dims[keep], axis=0, return_inverse=True)
        for gi, (na, nb) in enumerate(shapes):
            members = keep[group.reshape(-1) == gi]
            aa0, bb0 = np.meshgrid(np.arange(na), np.arange(nb), indexing="ij")
            aa0, bb0 = aa0.reshape(-1), bb0.reshape(-1)
            for c0 in range(0, len(members), chunk):
                m = members[c0:c0 + chunk]
                Ai, Aj, Ak = A[m, i][:, None], A[m, j][:, None], A[m, k][:, None]
                Bi, Bj, Bk = B[m, i][:, None], B[m, j][:, None], B[m, k][:, None]
                Ci, Cj, Ck = C[m, i][:, None], C[m, j][:, None], C[m, k][:, None]
                la = a0[m][:, None] + aa0[None, :]
                lb = b0[m][:, None] + bb0[None, :]
                pa, pb = la.astype(np.float64), lb.astype(np.float64)
                w0 = (Ci - Bi) * (pb - Bj) - (Cj - Bj) * (pa - Bi)
                w1 = (Ai - Ci) * (pb - Cj) - (Aj - Cj) * (pa - Ci)
                w2 = (Bi - Ai) * (pb - Aj) - (Bj - Aj) * (pa - Ai)
                ws = w0 + w1 + w2
                hit = (((w0 >= 0) & (w1 >= 0) & (w2 >= 0)) | ((w0 <= 0) & (w1 <= 0) & (w2 <= 0))) & (ws != 0)
                with np.errstate(divide="ignore", invalid="ignore"):
                    z = np.floor((w0 * Ak + w1 * Bk + w2 * Ck) / np.where(ws != 0, ws, 1.0))
                ok = hit & (z >= 0) & (z <= R - 2)
                q = [None, None, None]
                q[k], q[i], q[j] = z[ok].astype(np.int64), la[ok], lb[ok]
                blk[k, (q[2] * R + q[1]) * R + q[0]] = True
    return blk.reshape(3, R, R, R)


def outside_nodes(blk, R):
    """Nodes reachable from the grid's boundary through uncrossed edges."""
    out = np.zeros((R, R, R), bool)
    out[0, :, :] = out[-1, :, :] = out[:, 0, :] = out[:, -1, :] = out[:, :, 0] = out[:, :, -1] = True
    axis_of = {0: 2, 1: 1, 2: 0}                           # grid axis k -> array axis of [z, y, x]
    while True:
        before = out.sum()
        for k in range(3):
            ax = axis_of[k]
            o = np.moveaxis(out, ax, 0)
            b = np.moveaxis(blk[k], ax, 0)
            for c in range(1, R):
                o[c] |= o[c - 1] & ~b[c - 1]
            for c in range(R - 2, -1, -1):
                o[c] |= o[c + 1] & ~b[c]
        if out.sum() == before:
            return out


def field(d2, outside):
    far = d2 == FAR_D2
    u = np.where(far, 1e9, np.sqrt(d2.astype(np.float64)))
    return (np.where(outside, u, -u) - SHIFT_CELLS).astype(np.float32)


def contour(sd, R, table=None):
    """Marching cubes of sd < 0: (grid-unit vertices float64, tris int32).
    Vertices: one per crossed grid edge in edge-id order (3 * node + axis),
    then the centres of the loops longer than three, by cell (x fastest)
    and loop.  Triangles: by cell, loop and fan order."""
    loops = table or mc_case_table()
    inside = sd < 0
    # vertices on crossed grid edges, ordered by edge id 3 * node + axis
    ids = np.full((R, R, R, 3), -1, np.int64)             # [z, y, x, axis]
    verts = []
    flat = []
    for k, ax in ((0, 2), (1, 1), (2, 0)):
        sl0 = [slice(None)] * 3
        sl1 = [slice(None)] * 3
        sl0[ax] = slice(0, R - 1)
        sl1[ax] = slice(1, R)
        diff = np.zeros((R, R, R), bool)
        diff[tuple(sl0)] = inside[tuple(sl0)] != inside[tuple(sl1)]
        for z, y, x in zip(*np.nonzero(diff)):
            flat.append((((z * R + y) * R + x) * 3 + k, (x, y, z), k))
    flat.sort()
    for vid, (eid, (x, y, z), k) in enumerate(flat):
        ids[z, y, x, k] = vid
        n = [x, y, z]
        n1 = list(n)
        n1[k] += 1
        s0 = np.float64(sd[z, y, x])
        s1 = np.float64(sd[n1[2], n1[1], n1[0]])
        t = s0 / (s0 - s1)
        t = min(max(t, T_CLAMP), 1.0 - T_CLAMP)
        p = [float(x), float(y), float(z)]
        p[k] = p[k] + t
        verts.append(p)
    tris, centres = [], []
    nedge = len(verts)
    for z in range(R - 1):
        for y in range(R - 1):
            for x in range(R - 1):
                case = 0
                for c in range(8):
                    if inside[z + (c >> 2 & 1), y + (c >> 1 & 1), x + (c & 1)]:
                        case |= 1 << c
                for poly in loops[case]:
                    vid = []
                    for e in poly:
                        c0, _, k = EDGES[e]
                        vid.append(ids[z + (c0 >> 2 & 1), y + (c0 >> 1 & 1), x + (c0 & 1), k])
                    if len(vid) == 3:
                        tris.append(vid)
                        continue
                    cx = cy = cz = 0.0
                    for q in vid:
                        cx += verts[q][0]; cy += verts[q][1]; cz += verts[q][2]
                    m = float(len(vid))
                    centre = nedge + len(centres)
                    centres.append([cx / m, cy / m, cz / m])
                    for i in range(len(vid)):
                        tris.append([centre, vid[i], vid[(i + 1) % len(vid)]])
    allv = np.asarray(verts + centres, np.float64).reshape(-1, 3)
    return allv, np.asarray(tris, np.int32).reshape(-1, 3)


def remesh(verts, tris, R):
    """(verts float32, tris int32) of the remeshed surface."""
    if R < 8 or R & (R - 1):
        raise ValueError("resolution must be a power of two >= 8")
    u, vmin, extent, band, margin = normalise(verts, R)
    if not extent > 0:
        raise ValueError("the mesh has no extent")
    d2 = distance_grid(u, tris, R)
    out = outside_nodes(crossed_edges(u, tris, R), R)
    sd = field(d2, out)
    gv, gt = contour(sd, R)
    p = ((gv + 0.5) / R * margin - band) * np.float64(extent) + vmin.astype(np.float64)
    return p.astype(np.float32), gt
