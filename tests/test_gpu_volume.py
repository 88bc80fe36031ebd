"""GPU batched mesh volume vs the FP64 oracle (1e-5 relative)."""
import numpy as np
import pytest

from conftest import box_mesh
from cuacd_b200 import workloads as W

pytestmark = pytest.mark.gpu
VOL_RTOL = 1e-5


def test_known_and_batch(ctx, oracle):
    meshes = [box_mesh([0, 0, 0], [1, 1, 1])] + [W.icosphere(l) for l in (1, 3, 5)]
    meshes += [W.candidate_mesh(), W.hausdorff_sphere(4)]
    vs = [m[0].astype(np.float32) for m in meshes]
    ts = [m[1] for m in meshes]
    out = ctx.batch_mesh_volume(vs, ts)
    assert abs(out[0] - 1.0) < 1e-6
    for o, v, t in zip(out, vs, ts):
        ref = oracle.mesh_volume(v, t)
        assert abs(o - ref) / ref < VOL_RTOL


def test_uneven_many(ctx, oracle):
    rng = np.random.default_rng(3)
    meshes = []
    for i in range(40):
        lvl = int(rng.integers(0, 5))
        v, t = W.icosphere(lvl)
        v = (v * rng.uniform(0.2, 2.0) + rng.uniform(-3, 3, 3)).astype(np.float32)
        meshes.append((v, t))
    out = ctx.batch_mesh_volume([m[0] for m in meshes], [m[1] for m in meshes])
    for o, (v, t) in zip(out, meshes):
        ref = oracle.mesh_volume(v, t)
        assert abs(o - ref) / ref < VOL_RTOL
