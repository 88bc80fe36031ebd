"""gpu_mesh_audit (Context.check_mesh) against the reference's own GPU
verdicts and against the oracle on randomly broken meshes."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from ref_gpu_cases import M

pytestmark = pytest.mark.gpu
REF = os.path.join(GOLDEN, "ref_gpu_audit.npz")


@pytest.mark.skipif(not os.path.exists(REF), reason="no recorded reference verdicts")
def test_matches_reference_verdicts(ctx):
    ref = np.load(REF)
    for name, v, t in M.audit_cases():
        r = ctx.check_mesh(v, t)
        assert r["flags"] == int(ref[name][0]), name
        assert r["needs_remesh"] == bool(r["flags"])


def test_random_breakage_matches_oracle(ctx, oracle):
    rng = np.random.default_rng(31)
    v, t = M.W.candidate_mesh(32, 12, 0.35, seed=3)
    t = t.astype(np.int32)
    for trial in range(40):
        tt = t.copy()
        kind = trial % 5
        k = rng.integers(1, 4)
        rows = rng.choice(len(tt), k, replace=False)
        if kind == 0:
            tt = np.delete(tt, rows, axis=0)
        elif kind == 1:
            tt[rows] = tt[rows][:, [0, 2, 1]]
        elif kind == 2:
            tt = np.concatenate([tt, tt[rows]])
        elif kind == 3:
            tt[rows, 1] = tt[rows, 0]
        else:
            tt[rows, 2] = len(v) + rng.integers(0, 5)
        assert ctx.check_mesh(v, tt)["flags"] == oracle.mesh_audit(v, tt), (trial, kind)


def test_closed_meshes_pass(ctx):
    for v, t in [M.W.candidate_mesh(), M.W.hausdorff_sphere(level=4)]:
        r = ctx.check_mesh(v, t)
        assert r["watertight"] and r["manifold"] and r["oriented"] and not r["needs_remesh"]
    assert ctx.check_mesh(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32))["flags"] == 0
