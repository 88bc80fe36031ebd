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
