"""Shared fixtures.  Tests marked `gpu` need a CUDA device (B200); the rest
run on the CPU (oracle pins, host logic, library load/exports)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def ctx():
    import cuacd_b200
    c = cuacd_b200.Context(0)
    yield c
    c.close()


def box_mesh(lo, hi):
    """Closed box as 8 vertices / 12 triangles with outward winding."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float32)
    t = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [2, 3, 7], [2, 7, 6], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]], np.int32)
    return v, t


def l_shape():
    v1, t1 = box_mesh([0, 0, 0], [1, 1, 1])
    v2, t2 = box_mesh([1, 0, 0], [2, 1, 0.5])
    return np.vstack([v1, v2]), np.vstack([t1, t2 + len(v1)])


def torus_mesh(R, r, nu=48, nv=16):
    """Closed torus around the z axis (nu x nv grid), outward winding."""
    u = np.arange(nu) * (2 * np.pi / nu)
    w = np.arange(nv) * (2 * np.pi / nv)
    U, V = np.meshgrid(u, w, indexing="ij")
    verts = np.stack([(R + r * np.cos(V)) * np.cos(U), (R + r * np.cos(V)) * np.sin(U), r * np.sin(V)], -1)
    idx = lambda i, j: (i % nu) * nv + (j % nv)
    tris = []
    for i in range(nu):
        for j in range(nv):
            a, b, c, d = idx(i, j), idx(i + 1, j), idx(i + 1, j + 1), idx(i, j + 1)
            tris += [(a, b, c), (a, c, d)]
    v = verts.reshape(-1, 3).astype(np.float32)
    t = np.asarray(tris, np.int32)
    e = v[t]
    if np.einsum("ij,ij->i", e[:, 0], np.cross(e[:, 1], e[:, 2])).sum() < 0:
        t = t[:, ::-1].copy()
    return v, t


def nested_tori():
    """Three concentric tori (R = 1, 2, 3; r = 0.3): a cut across their ring
    gives six nested circles, annuli inside annuli."""
    parts = [torus_mesh(R, 0.3) for R in (1.0, 2.0, 3.0)]
    v = np.concatenate([p[0] for p in parts])
    offs = np.cumsum([0] + [len(p[0]) for p in parts[:-1]])
    t = np.concatenate([p[1] + o for p, o in zip(parts, offs)]).astype(np.int32)
    return v, t


def box_with_cavity():
    """Unit box holding an inverted inner box (a closed cavity)."""
    a = box_mesh([0, 0, 0], [1, 1, 1])
    b = box_mesh([0.3, 0.3, 0.3], [0.7, 0.7, 0.7])
    return np.vstack([a[0], b[0]]).astype(np.float32), np.vstack([a[1], b[1][:, ::-1] + 8]).astype(np.int32)


def is_watertight(t):
    """Every directed edge has exactly one reverse partner."""
    t = np.asarray(t)
    if len(t) == 0:
        return False
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    fwd = {}
    for a, b in e.tolist():
        fwd[(a, b)] = fwd.get((a, b), 0) + 1
    return all(fwd.get((b, a), 0) == c for (a, b), c in fwd.items())
