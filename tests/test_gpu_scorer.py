"""The learned scorer's GPU kernels against the FP64 numpy restatement
(oracle/scorer_ref.py): feature rows, BF16 tensor-core forward and backward
(gradient check), AdamW; training reduces the loss; the pruned evaluator
returns exact results for every plane it evaluates; and (with the trained
weights) the network's top-8 beats random top-8."""
import os

import numpy as np
import pytest

from cuacd_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def S():
    from cuacd_b200 import scorer
    return scorer


@pytest.fixture(scope="module")
def ref():
    from oracle import scorer_ref
    return scorer_ref


@pytest.fixture(scope="module")
def part():
    v, t = W.candidate_mesh(48, 16, 0.35, seed=5)
    return v, t


def test_features_match_fp64(ctx, S, ref, part):
    v, t = part
    sc = S.Scorer(ctx, seed=1)
    planes = S.candidate_set(ctx, v, t)
    assert len(planes) >= 8
    hv = S.part_hull_volume(ctx, v)
    got = sc.features(v, t, planes, hv)
    want = ref.features(v, t, planes, hv)
    assert got.shape == want.shape == (len(planes), 240)
    hist = slice(54, 70)
    other = np.r_[0:54, 70:240]
    # FP32 block sums over a few thousand vertices: 1e-4 absolute in R units
    np.testing.assert_allclose(got[:, other], want[:, other], atol=2e-4, rtol=1e-4)
    # a vertex on a bin edge may fall either side in FP32
    assert np.abs(got[:, hist] - want[:, hist]).max() <= 2.0 / len(v) + 1e-7
    assert np.all(got[:, 230:] == 0)


def _rows(ctx, S, part, n_extra=0):
    v, t = part
    sc = S.Scorer(ctx, seed=2)
    planes = S.candidate_set(ctx, v, t)
    X = sc.features(v, t, planes, S.part_hull_volume(ctx, v))
    rng = np.random.default_rng(0)
    if n_extra:
        X = np.concatenate([X, X[rng.integers(0, len(X), n_extra)] + rng.normal(0, 0.05, (n_extra, 240)).astype(np.float32)])
        X[:, 230:] = 0
    T = rng.uniform(0.0, 0.3, len(X)).astype(np.float32)
    return sc, X, T


def test_gradient_check(ctx, S, ref, part):
    sc, X, T = _rows(ctx, S, part, n_extra=70)
    p = sc.params()
    loss, g = sc.grad(X, T)
    rloss, rg = ref.loss_grad(p, X, T)
    assert abs(loss - rloss) <= 2e-2 * rloss + 1e-6
    gd, rd = ref.unpack(g), ref.unpack(rg)
    for name in ("W1", "b1", "W2", "b2", "W3", "b3"):
        a, b = gd[name].ravel(), rd[name].ravel()
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        cos = a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30)
        # BF16 operands (8-bit mantissa), FP32 accumulation
        assert rel < 3e-2, (name, rel)
        assert cos > 0.999, (name, cos)


def test_forward_matches_fp64(ctx, S, ref, part):
    sc, X, _ = _rows(ctx, S, part, n_extra=30)
    y = sc.predict(X)
    ry = ref.forward(sc.params(), X)[0] / ref.TSCALE
    assert np.abs(y - ry).max() <= 2e-2 * np.abs(ry).max() + 1e-4


def test_normalizer_applied(ctx, S, ref, part):
    sc, X, _ = _rows(ctx, S, part, n_extra=10)
    rng = np.random.default_rng(3)
    mean = X.mean(0).astype(np.float32)
    inv = (1.0 / (X.std(0) + 0.1)).astype(np.float32)
    sc.set_normalizer(mean, inv)
    m2, i2 = sc.normalizer()
    np.testing.assert_array_equal(m2, mean)
    np.testing.assert_array_equal(i2, inv)
    y = sc.predict(X)
    ry = ref.forward(sc.params(), X, mean, inv)[0] / ref.TSCALE
    assert np.abs(y - ry).max() <= 2e-2 * np.abs(ry).max() + 1e-4


def test_adamw_step_matches_fp64(ctx, S, ref, part):
    sc, X, T = _rows(ctx, S, part, n_extra=34)
    n = len(X)
    p0 = sc.params()
    _, g = sc.grad(X, T)
    lr, wd = 1e-3, 0.01
    sc.train(X, T, epochs=1, batch=n, lr=lr, wd=wd, seed=0)
    p1 = sc.params()
    want, _, _ = ref.adamw_step(p0, g, np.zeros(len(p0)), np.zeros(len(p0)), 1, lr, wd)
    # the step moves each parameter by about lr; a gradient element whose
    # sign differs between two FP32 summation orders may move the other way
    close = np.abs(p1 - want) <= 0.05 * lr + 1e-7
    assert close.mean() > 0.999
    assert np.abs(p1 - p0).max() <= 1.01 * lr * (1 + wd * np.abs(p0).max()) + 1e-6


def test_training_reduces_loss(ctx, S, part):
    v, t = part
    sc = S.Scorer(ctx, seed=3)
    X, T, G = S.build_dataset(ctx, sc, [(v, t), W.candidate_mesh(32, 12, 0.3, seed=9)])
    l0 = float(np.mean((sc.predict(X) - T) ** 2))
    l1 = sc.train(X, T, epochs=200, batch=32, lr=1e-3, wd=0.0, seed=1)
    l2 = float(np.mean((sc.predict(X) - T) ** 2))
    assert l1 < 0.3 * l0 and l2 < 0.3 * l0, (l0, l1, l2)


def test_pruned_exact_on_evaluated(ctx, S, part):
    v, t = part
    sc = S.Scorer(ctx, seed=4)
    planes = S.candidate_set(ctx, v, t)
    exact = ctx.eval_candidates(v, t, planes)
    res, pred, ev = sc.eval_pruned(v, t, planes, top_k=8)
    assert ev.sum() >= 8
    order = np.argsort(pred, kind="stable")
    assert set(order[:8]) <= set(np.nonzero(ev)[0])
    for i in range(len(planes)):
        if ev[i]:
            assert res[i] == exact[i]
        else:
            assert res[i]["ok"] == 0 and res[i]["score_full"] > 1e38
    # a margin wider than any prediction gap sends every plane to the exact path
    res2, _, ev2 = sc.eval_pruned(v, t, planes, top_k=1, margin=1e9)
    assert ev2.all() and res2 == exact


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                    "cuacd_b200", "scorer_weights.npz")),
                    reason="no trained weights")
def test_ablation_trained_vs_random(ctx, S):
    """What the trained network gains: on held-out parts (seeds unseen in
    training) its top-8 of the level's planes contains the exact best plane
    far more often than 8 random planes, and the best exact score within
    its top-8 is closer to the true best."""
    sc = S.Scorer.load(ctx)
    X, T, G = S.build_dataset(ctx, sc, S.training_meshes(24, 777))
    hit, reg, rreg = S.ranking_quality(sc.predict(X), T, G)
    sizes = np.bincount(G)
    random_hit = float(np.mean(np.minimum(8, sizes) / sizes))
    assert hit > random_hit + 0.15, (hit, random_hit)
    assert reg < 0.5 * rreg, (reg, rreg)


def test_pruned_device_matches_host(ctx, S, part):
    """The device-pointer pruned evaluation (selection and scatter on the
    GPU) returns the host entry point's results, predictions and mask."""
    import ctypes
    import torch
    import cuacd_b200
    v, t = part
    sc = S.Scorer(ctx, seed=4)
    planes = S.candidate_set(ctx, v, t)
    n = len(planes)
    hv = S.part_hull_volume(ctx, v)
    res, pred, ev = sc.eval_pruned(v, t, planes, top_k=5, margin=0.01, hull_vol=hv)
    dv = torch.from_numpy(v.reshape(-1)).cuda()
    dt = torch.from_numpy(t.reshape(-1).astype(np.int32)).cuda()
    dp = torch.from_numpy(planes.reshape(-1)).cuda()
    nb = ctypes.sizeof(cuacd_b200.CandResult) * n
    dout = torch.zeros(nb, dtype=torch.uint8, device="cuda")
    dpred = torch.zeros(n, dtype=torch.float32, device="cuda")
    dev = torch.zeros(n, dtype=torch.int32, device="cuda")
    ne = ctypes.c_int(0)
    stream = torch.cuda.current_stream()
    rc = cuacd_b200._fn("cuacd_eval_candidates_pruned_device")(
        ctx.handle, sc._h, ctypes.c_void_p(dv.data_ptr()), len(v), ctypes.c_void_p(dt.data_ptr()), len(t),
        float(hv), ctypes.c_void_p(dp.data_ptr()), n, 1, 2000.0, 1000, 0, 5, 0.01,
        ctypes.c_void_p(dout.data_ptr()), ctypes.c_void_p(dpred.data_ptr()), ctypes.c_void_p(dev.data_ptr()),
        ctypes.byref(ne), ctypes.c_void_p(stream.cuda_stream))
    ctx._check(rc)
    torch.cuda.synchronize()
    host = (cuacd_b200.CandResult * n)()
    buf = dout.cpu().numpy()
    ctypes.memmove(host, buf.ctypes.data, nb)
    got = [cuacd_b200.cand_to_dict(r) for r in host]
    assert ne.value == int(ev.sum())
    np.testing.assert_array_equal(dev.cpu().numpy().astype(bool), ev)
    np.testing.assert_array_equal(dpred.cpu().numpy(), pred)
    assert got == res


def test_search_scorer_ranks_level0(ctx, S):
    """The trained level-0 scorer on held-out parts (seeds unseen in
    training), over the search's level-0 planes (32 concave edges, 30 axis
    cuts): its top 48 contains the plane with the lowest exact rv cost far
    more often than 48 random planes do."""
    sc = S.Scorer.load(ctx, S.RV_WEIGHTS_PATH)
    plane_set = {"n_concave_edges": 32, "width": 30, "max_concave": 128}
    X, T, G = S.build_dataset(ctx, sc, S.training_meshes(12, 4242), plane_set=plane_set, target="rv")
    hit, reg, rreg = S.ranking_quality(sc.predict(X), T, G, k=48)
    sizes = np.bincount(G)
    random_hit = float(np.mean(np.minimum(48, sizes) / sizes))
    assert hit > random_hit + 0.3, (hit, random_hit)
    assert reg < 0.25 * rreg, (reg, rreg)


def test_forward_stages_activations_by_tma(ctx, S, ref):
    """A forward pass of 300 rows: every layer's A operand (the feature rows,
    then the hidden activations) is a K-major contiguous matrix, so its
    slabs reach shared memory by TMA (128-byte swizzle), and the output
    still matches the FP64 forward of the same BF16 parameters."""
    import ctypes
    from cuacd_b200 import _fn
    counts = lambda: [ctypes.c_ulonglong(0), ctypes.c_ulonglong(0)]
    a0, s0 = counts()
    _fn("cuacd_scorer_gemm_counts")(ctypes.byref(a0), ctypes.byref(s0))
    X = np.random.default_rng(11).standard_normal((300, S.N_FEATURES)).astype(np.float32)
    with S.Scorer(ctx, seed=3) as sc:
        y = sc.predict(X)
        mean, inv = sc.normalizer()
        params = sc.params()
    a1, s1 = counts()
    _fn("cuacd_scorer_gemm_counts")(ctypes.byref(a1), ctypes.byref(s1))
    assert a1.value - a0.value == 3 and s1.value == s0.value
    ry = ref.forward(params, X, mean, inv)[0] / ref.TSCALE
    assert np.abs(y - ry).max() <= 2e-2 * np.abs(ry).max() + 1e-3
