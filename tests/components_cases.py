"""Meshes for the connected-components tests (shared by the CPU oracle pins
and the GPU parity tests).  The first six follow the cases of the
reference's tests/test_decompose_components.py."""
import numpy as np

from conftest import box_mesh


def cube(center=(0, 0, 0), size=1.0):
    c = np.asarray(center, np.float32)
    h = np.float32(size / 2)
    return box_mesh(c - h, c + h)


def tetrahedron(center=(0, 0, 0), size=1.0):
    cx, cy, cz = center
    s = size
    v = np.array([[cx + s, cy + s, cz + s], [cx + s, cy - s, cz - s],
                  [cx - s, cy + s, cz - s], [cx - s, cy - s, cz + s]], np.float32)
    t = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.int32)
    return v, t


def merge(meshes):
    vs, ts, off = [], [], 0
    for v, t in meshes:
        vs.append(np.asarray(v, np.float32))
        ts.append(np.asarray(t, np.int32) + off)
        off += len(v)
    return np.concatenate(vs).astype(np.float32), np.concatenate(ts).astype(np.int32)


def shared_face_cubes():
    """Two cubes sharing four vertices: one component."""
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                  [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1],
                  [2, 0, 0], [2, 1, 0], [2, 0, 1], [2, 1, 1]], np.float32)
    t = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [2, 3, 7], [2, 7, 6], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5],
                  [1, 9, 8], [1, 2, 9], [5, 10, 11], [5, 11, 6], [1, 8, 10], [1, 10, 5],
                  [9, 2, 6], [9, 6, 11], [1, 5, 6], [1, 6, 2], [8, 9, 11], [8, 11, 10]], np.int32)
    return v, t


def inverted(mesh):
    v, t = mesh
    return v, t[:, ::-1].copy()


def shuffled(mesh, seed):
    """Same mesh with vertices and triangles in random order."""
    v, t = mesh
    rng = np.random.default_rng(seed)
    pv = rng.permutation(len(v))
    inv = np.empty_like(pv)
    inv[pv] = np.arange(len(v))
    v2 = v[pv]
    t2 = inv[t][rng.permutation(len(t))]
    return v2.astype(np.float32), t2.astype(np.int32)


def many_boxes(n, seed, spacing=3.0):
    rng = np.random.default_rng(seed)
    ms = []
    for i in range(n):
        c = np.array([i % 17, (i // 17) % 17, i // 289], np.float32) * spacing + rng.uniform(-0.2, 0.2, 3)
        ms.append(cube(c, float(rng.uniform(0.5, 1.5))))
    return merge(ms)


def shells_with_cavities(seed):
    """Outer boxes with inverted inner boxes (cavities) and a stray vertex."""
    rng = np.random.default_rng(seed)
    ms = []
    for i in range(6):
        c = np.array([4.0 * i, 0, 0], np.float32)
        ms.append(cube(c, 2.0))
        if i % 2 == 0:
            ms.append(inverted(cube(c + rng.uniform(-0.1, 0.1, 3), 0.8)))
    v, t = merge(ms)
    v = np.vstack([v, np.array([[50, 50, 50]], np.float32)])      # used by no triangle
    return v, t


def cases():
    """(name, verts, tris) for the parity tests."""
    return [
        ("single_cube", *cube()),
        ("two_cubes", *merge([cube((0, 0, 0)), cube((5, 0, 0))])),
        ("three_tets", *merge([tetrahedron((0, 0, 0)), tetrahedron((10, 0, 0)), tetrahedron((0, 10, 0))])),
        ("shared_face", *shared_face_cubes()),
        ("volume_pair", *merge([cube((0, 0, 0), 2.0), cube((10, 0, 0), 3.0)])),
        ("cubes_33", *merge([cube((3 * i, 0, 0)) for i in range(33)])),
        ("all_inner", *merge([inverted(cube((0, 0, 0))), inverted(cube((4, 0, 0)))])),
        ("cavities", *shells_with_cavities(5)),
        ("shuffled_boxes", *shuffled(many_boxes(40, 1), 7)),
    ]
