"""The command line on the GPU: an OBJ file in, a GLB of convex parts out,
through the real context, in serial mode and through the spawned pipeline.
The GLB must hold exactly the hulls that Context.lookahead_decompose gives
for the loaded mesh with the command's default options, after the
command's normalisation (centre of the bounding box, half the longest
side) is undone.  The input is two boxes meeting along an edge: loading
merges their two shared corners, so they form one non-manifold component,
which the audit flags -- by default the command remeshes it first
(Context.preprocess at resolution 64), with --preprocess off it does not."""
import numpy as np
import pytest

from conftest import l_shape
from cuacd_b200 import cli, meshio

pytestmark = pytest.mark.gpu

CLI_DEFAULTS = dict(max_iters=100, width=30, width2=5, depth=2, quick_depth=0, threshold=0.05,
                    decompose_components=True, no_decompose_components_per_iter=False, n_concave_edges=16,
                    concave_eps=0.005, concave_threshold=3.49, concave_iters=10, merge_hulls=True)


def _volume(v, t):
    v = v.astype(np.float64)
    return float(np.einsum("ij,ij->i", v[t[:, 0]], np.cross(v[t[:, 1]], v[t[:, 2]])).sum() / 6.0)


@pytest.mark.parametrize("mode", [["--serial"], [], ["--serial", "--preprocess", "off"]])
def test_cli_matches_the_library(ctx, tmp_path, mode, capfd):
    v, t = l_shape()
    src = tmp_path / "in"
    src.mkdir()
    (src / "ell.obj").write_text("\n".join([f"v {x!r} {y!r} {z!r}" for x, y, z in v.tolist()] +
                                           [f"f {a + 1} {b + 1} {c + 1}" for a, b, c in t.tolist()]) + "\n")
    out = tmp_path / "out"
    rc = cli.main([str(src), str(out)] + mode)
    so, se = capfd.readouterr()
    assert rc == 0, se
    got = meshio.read_glb_parts((out / "ell.glb").read_bytes())

    lv, lt = meshio.load_mesh(src / "ell.obj")
    assert len(lv) == 14                                   # 16 corners, 2 shared
    audit = ctx.check_mesh(lv, lt)
    assert audit["needs_remesh"]
    if "off" not in mode:
        lv, lt = ctx.preprocess(lv, lt, resolution=64)
    lo, hi = lv.min(axis=0), lv.max(axis=0)
    center = (lo + hi) / 2
    scale = float((hi - lo).max()) / 2
    parts = ctx.lookahead_decompose(((lv - center) / scale).astype(np.float32), lt, **CLI_DEFAULTS)
    want = [(hv * scale + center, ht) for _, _, hv, ht in parts]
    assert [g[0] for g in got] == [f"ell_{i}" for i in range(len(want))]
    for (_, gv, gt, col), (wv, wt) in zip(got, want):
        np.testing.assert_array_equal(gv, np.asarray(wv, np.float32))
        np.testing.assert_array_equal(gt, wt)
        assert col is not None and col[3] == 255
    assert sum(_volume(gv, gt) for _, gv, gt, _ in got) >= _volume(lv, lt) * (1 - 1e-6)
    assert "ell.obj" in so and f"{len(want)} parts" in so
