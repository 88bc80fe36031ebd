"""The hull pipeline's launch-shape tuning (cuacd_b200/autotune.py):
settings round-trip per size class, a short sweep picks one of the timed
shapes, and every shape gives bit-identical hulls (the sweep itself checks
this and raises otherwise; here it is also checked against the oracle)."""
import numpy as np
import pytest

from cuacd_b200 import autotune as AT
from cuacd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_set_get_round_trip(ctx):
    old = [AT.get_tuning(ctx, c) for c in AT.CLASSES]
    try:
        AT.set_tuning(ctx, 1, 2048, 4096)
        assert AT.get_tuning(ctx, 1) == (2048, 4096)
        AT.set_tuning(ctx, 1, 0, 0)                     # defaults
        assert AT.get_tuning(ctx, 1) == (4096, 1 << 30)
    finally:
        for c, (p, s) in zip(AT.CLASSES, old):
            AT.set_tuning(ctx, c, p, s)


def test_short_sweep_and_shape_invariance(ctx, oracle):
    old = [AT.get_tuning(ctx, c) for c in AT.CLASSES]
    rng = np.random.default_rng(5)
    shell = []
    for n in (6000, 9000):
        d = rng.normal(size=(n, 3))
        shell.append((d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32))
    big = rng.normal(size=(70000, 3))
    big = (big / np.linalg.norm(big, axis=1, keepdims=True) * rng.uniform(0.97, 1.0, (70000, 1))).astype(np.float32)
    batches = {0: W.hull_clouds(32, 1000, 0), 1: shell, 2: [big]}
    try:
        res = AT.tune(ctx, reps=1, pts_per_cta=(2048, 8192), seed_min_n={0: (0,), 1: (0, 4096), 2: (0, 65536)},
                      batches=batches)
        assert len(res["hull"]) == 3
        for c, (ppc, seed) in enumerate(res["hull"]):
            assert ppc in (2048, 8192) and AT.get_tuning(ctx, c)[0] == ppc
        for c in (1, 2):
            AT.set_tuning(ctx, c, 2048, 1)              # six seeds for every cloud
        for cloud in shell + [big]:
            (hv, ht, vol), = ctx.batch_hull_dandc_mesh([cloud])
            idx, tris, ovol = oracle.hull(cloud)
            np.testing.assert_array_equal(hv, cloud[idx])
            np.testing.assert_array_equal(ht, tris)
    finally:
        for c, (p, s) in zip(AT.CLASSES, old):
            AT.set_tuning(ctx, c, p, s)
