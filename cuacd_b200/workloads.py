"""Seeded synthetic workloads for the candidate-evaluation path.

Every mesh here is closed, consistently wound (outward normals) and built
from seeded numpy random state, so a workload is reproduced exactly from its
name and seed.  These stand in for the reference's public datasets, which are
not part of this build.
"""
import numpy as np


# ---------------------------------------------------------------------------
# base meshes
# ---------------------------------------------------------------------------

def icosphere(level):
    """Unit icosphere: regular icosahedron with `level` rounds of 4-way
    midpoint subdivision (20*4**level triangles)."""
    g = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, g, 0), (1, g, 0), (-1, -g, 0), (1, -g, 0),
         (0, -1, g), (0, 1, g), (0, -1, -g), (0, 1, -g),
         (g, 0, -1), (g, 0, 1), (-g, 0, -1), (-g, 0, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
             (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
             (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
             (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        mid = {}

        def midpoint(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in mid:
                p = verts[a] + verts[b]
                verts.append(p / np.linalg.norm(p))
                mid[key] = len(verts) - 1
            return mid[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts, dtype=np.float64), np.array(faces, dtype=np.int32)


def uv_sphere(n_lon, n_rings):
    """Unit UV sphere with two poles and `n_rings` vertex rings of `n_lon`
    vertices: 2 + n_lon*n_rings vertices, 2*n_lon*n_rings triangles."""
    th = np.pi * (np.arange(n_rings) + 1) / (n_rings + 1)
    ph = 2 * np.pi * np.arange(n_lon) / n_lon
    T, P = np.meshgrid(th, ph, indexing="ij")
    ring = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1).reshape(-1, 3)
    verts = np.concatenate([[[0, 0, 1]], ring, [[0, 0, -1]]]).astype(np.float64)
    top, bot = 0, len(verts) - 1
    idx = lambda r, k: 1 + r * n_lon + (k % n_lon)
    tris = []
    for k in range(n_lon):
        tris.append((top, idx(0, k), idx(0, k + 1)))
    for r in range(n_rings - 1):
        for k in range(n_lon):
            a, b = idx(r, k), idx(r, k + 1)
            c, d = idx(r + 1, k), idx(r + 1, k + 1)
            tris.append((a, c, b))
            tris.append((b, c, d))
    for k in range(n_lon):
        tris.append((bot, idx(n_rings - 1, k + 1), idx(n_rings - 1, k)))
    return verts, np.array(tris, dtype=np.int32)


def box(lo, hi, subdiv=1):
    """Axis-aligned box [lo, hi] with each face split into subdiv x subdiv
    quads (2 triangles each), outward winding, shared vertices."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    n = int(subdiv)
    g = np.linspace(0.0, 1.0, n + 1)
    verts = {}
    out_v = []

    def vid(p):
        key = tuple(np.round(p, 12))
        if key not in verts:
            verts[key] = len(out_v)
            out_v.append(p)
        return verts[key]

    tris = []
    # each face: fixed axis, side, and two in-face axes ordered for outward winding
    for axis in range(3):
        u, w = (axis + 1) % 3, (axis + 2) % 3
        for side in (0, 1):
            grid = np.empty((n + 1, n + 1), dtype=np.int64)
            for i in range(n + 1):
                for j in range(n + 1):
                    p = np.empty(3)
                    p[axis] = hi[axis] if side else lo[axis]
                    p[u] = lo[u] + g[i] * (hi[u] - lo[u])
                    p[w] = lo[w] + g[j] * (hi[w] - lo[w])
                    grid[i, j] = vid(p)
            for i in range(n):
                for j in range(n):
                    a, b, c, d = grid[i, j], grid[i + 1, j], grid[i + 1, j + 1], grid[i, j + 1]
                    if side:
                        tris += [(a, b, c), (a, c, d)]
                    else:
                        tris += [(a, c, b), (a, d, c)]
    return np.array(out_v, dtype=np.float64), np.array(tris, dtype=np.int32)


# ---------------------------------------------------------------------------
# displacement fields
# ---------------------------------------------------------------------------

def _sine_field(pts, rng, n_terms, fmin, fmax):
    """Sum of random oriented low-frequency sines, scaled to [-1, 1]."""
    dirs = rng.standard_normal((n_terms, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    freq = rng.uniform(fmin, fmax, n_terms)
    phase = rng.uniform(0, 2 * np.pi, n_terms)
    amp = rng.uniform(0.5, 1.0, n_terms)
    f = (np.sin((pts @ dirs.T) * freq + phase) * amp).sum(1)
    return f / amp.sum()


def _ridged_field(pts, rng, n_terms, fmin, fmax):
    """Sum of random oriented |sin| terms: smooth crests with sharp valleys,
    so the surface gets concave creases (edges whose dihedral angle exceeds
    the concave-edge threshold)."""
    dirs = rng.standard_normal((n_terms, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    freq = rng.uniform(fmin, fmax, n_terms)
    phase = rng.uniform(0, 2 * np.pi, n_terms)
    amp = rng.uniform(0.5, 1.0, n_terms)
    f = (np.abs(np.sin((pts @ dirs.T) * freq + phase)) * amp).sum(1)
    f = f - f.mean()
    return f / max(np.abs(f).max(), 1e-12)


def displaced_sphere(verts, tris, amplitude, seed, n_terms=8, fmin=1.0, fmax=4.0, ridged=False):
    """Radially displace a unit sphere: r = 1 + amplitude * field(p)."""
    rng = np.random.default_rng(seed)
    f = (_ridged_field if ridged else _sine_field)(verts, rng, n_terms, fmin, fmax)
    f = f / max(np.abs(f).max(), 1e-12)
    return verts * (1.0 + amplitude * f)[:, None], tris


def normalize_extent(verts, extent=2.0):
    """Centre the bounding box at the origin and scale its largest side to
    `extent` (the caller-side normalisation the decomposition expects)."""
    lo, hi = verts.min(0), verts.max(0)
    c = 0.5 * (lo + hi)
    s = extent / max((hi - lo).max(), 1e-12)
    return (verts - c) * s


# ---------------------------------------------------------------------------
# named workloads
# ---------------------------------------------------------------------------

def hull_clouds(n_clouds=256, n_points=1000, seed=0):
    """Uniform point clouds in [-1,1]^3 (float32), one array per cloud."""
    pts = np.random.default_rng(seed).uniform(-1, 1, (n_clouds, n_points, 3)).astype(np.float32)
    return [pts[i] for i in range(n_clouds)]


def hausdorff_sphere(level=5, amplitude=0.25, seed=1):
    """Icosphere (20*4**level triangles) radially displaced by a sum of 8
    random low-frequency sines."""
    v, t = icosphere(level)
    v, t = displaced_sphere(v, t, amplitude, seed, n_terms=8, fmin=1.0, fmax=3.0)
    return v.astype(np.float32), t


def candidate_mesh(n_lon=256, n_rings=80, amplitude=0.35, seed=2):
    """Radially displaced UV sphere (2*n_lon*n_rings triangles; 40,960 at the
    defaults) normalised to extent 2.  The displacement is a ridged field, so
    the surface carries concave creases for the concave-edge planes."""
    v, t = uv_sphere(n_lon, n_rings)
    v, t = displaced_sphere(v, t, amplitude, seed, n_terms=6, fmin=2.0, fmax=5.0, ridged=True)
    return normalize_extent(v).astype(np.float32), t


def _sample_boxes(n_boxes, rng):
    """Up to n_boxes disjoint random boxes (rejection sampled in [-1,1]^3)."""
    boxes = []
    for _ in range(200 * n_boxes):
        if len(boxes) == n_boxes:
            break
        c = rng.uniform(-0.7, 0.7, 3)
        h = rng.uniform(0.08, 0.35, 3)
        lo, hi = c - h, c + h
        if any(np.all(lo < b[1] + 0.02) and np.all(b[0] < hi + 0.02) for b in boxes):
            continue
        boxes.append((lo, hi))
    return boxes


def _boxes_mesh(boxes, target_tris):
    per = max(12, target_tris // max(len(boxes), 1))
    sub = max(1, int(round((per / 12.0) ** 0.5)))
    vs, ts, off = [], [], 0
    for lo, hi in boxes:
        v, t = box(lo, hi, sub)
        vs.append(v)
        ts.append(t + off)
        off += len(v)
    return np.concatenate(vs), np.concatenate(ts).astype(np.int32)


def random_boxes_mesh(n_boxes, target_tris, rng):
    """Union of n_boxes disjoint random boxes (rejection sampled in [-1,1]^3)
    as one multi-shell mesh with about target_tris triangles."""
    return _boxes_mesh(_sample_boxes(n_boxes, rng), target_tris)


def batch_meshes(n_meshes=512, tmin=500, tmax=200_000, seed=3, select=None):
    """Uneven batch: triangle counts log-uniform in [tmin, tmax]; even
    indices are displaced spheres, odd ones unions of 2-6 random boxes.
    All meshes are normalised to extent 2.  `select` (indices) builds only
    those meshes -- the random draws of the others are still made, so a
    selected mesh is the same as in the full batch."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_meshes):
        target = int(np.exp(rng.uniform(np.log(tmin), np.log(tmax))))
        keep = select is None or i in select
        if i % 2 == 0:
            lvl = max(1, int(round(np.log(max(target, 80) / 20.0) / np.log(4.0))))
            sd = int(rng.integers(1 << 30))
            if not keep:
                continue
            v, t = icosphere(min(lvl, 7))
            v, t = displaced_sphere(v, t, 0.3, sd)
        else:
            boxes = _sample_boxes(int(rng.integers(2, 7)), rng)
            if not keep:
                continue
            v, t = _boxes_mesh(boxes, target)
        out.append((normalize_extent(v).astype(np.float32), t))
    return out
