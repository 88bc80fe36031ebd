"""The mesh-audit oracle against the reference's own GPU verdicts
(tests/golden/ref_gpu_audit.npz, recorded on a B200 from eliphatfs/cuacd's
`_gpu.mesh_audit` by tests/golden/make_ref_gpu.py --audit) on closed meshes
and on the same meshes broken in each way the verdict bits name."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from ref_gpu_cases import M

REF = os.path.join(GOLDEN, "ref_gpu_audit.npz")


@pytest.mark.skipif(not os.path.exists(REF), reason="no recorded reference verdicts")
def test_oracle_matches_reference_verdicts(oracle):
    ref = np.load(REF)
    cases = M.audit_cases()
    assert sorted(ref.files) == sorted(c[0] for c in cases)
    for name, v, t in cases:
        assert oracle.mesh_audit(v, t) == int(ref[name][0]), name


def test_oracle_known_verdicts(oracle):
    v, t = M.W.box((0, 0, 0), (1, 1, 1), 1)
    assert oracle.mesh_audit(v, t) == 0
    assert oracle.mesh_audit(v, t[:-1]) == 4                    # open
    assert oracle.mesh_audit(v, t[:, [0, 2, 1]]) == 0           # every face flipped: still consistent
    f = t.copy(); f[0] = f[0][[0, 2, 1]]
    assert oracle.mesh_audit(v, f) == 16                        # one face flipped
    assert oracle.mesh_audit(v, np.zeros((0, 3), np.int32)) == 0
