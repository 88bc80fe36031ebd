"""Pins of the scorer's FP64 oracle (oracle/scorer_ref.py) on the CPU: its
analytic gradient matches central finite differences, AdamW's first step
moves each parameter by lr (plus decay), and the feature rows obey the
layout's invariants on a mesh with known geometry."""
import numpy as np

from conftest import box_mesh
from oracle import scorer_ref as R


def _params(rng, scale=0.1):
    n = R.K * R.H + R.H + R.H * R.H + R.H + R.H + 1
    p = rng.normal(0, scale, n)
    d = R.unpack(p)
    d["W1"][R.NF:] = 0
    return R.pack(d)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = _params(rng)
    X = rng.normal(0, 1, (6, R.K))
    X[:, R.NF:] = 0
    T = rng.uniform(0, 0.3, 6)
    _, g = R.loss_grad(p, X, T)
    idx = np.concatenate([rng.integers(0, len(p), 40), [len(p) - 1, R.K * R.H + 3]])
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (R.loss_grad(p + e, X, T)[0] - R.loss_grad(p - e, X, T)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_adamw_first_step():
    rng = np.random.default_rng(1)
    p = _params(rng)
    g = rng.normal(0, 1, len(p))
    lr, wd = 1e-3, 0.1
    p1, m, v = R.adamw_step(p, g, np.zeros_like(p), np.zeros_like(p), 1, lr, wd)
    d0, d1, dg = R.unpack(p), R.unpack(p1), R.unpack(g)
    # step 1: the bias-corrected moments are g and g^2, so the step is g / (|g| + eps)
    for name in ("W1", "W2", "W3"):
        step = dg[name] / (np.abs(dg[name]) + 1e-8)
        np.testing.assert_allclose(d1[name], d0[name] * (1 - lr * wd) - lr * step, atol=1e-12)
    for name in ("b1", "b2", "b3"):
        step = dg[name] / (np.abs(dg[name]) + 1e-8)
        np.testing.assert_allclose(d1[name], d0[name] - lr * step, atol=1e-12)


def test_features_layout_on_a_box():
    v, t = box_mesh([0, 0, 0], [2, 2, 2])
    planes = np.array([[1, 0, 0, -1], [0, 1, 0, -0.5]], np.float64)
    f = R.features(v, t, planes, hull_vol=8.0)
    R_ = np.sqrt(3.0)
    np.testing.assert_allclose(f[:, 36:39], 1.0)                    # centroid
    np.testing.assert_allclose(f[0, 3], 0.0, atol=1e-12)           # plane through the centroid
    np.testing.assert_allclose(f[0, 4], 0.5)                       # half the vertices each side
    np.testing.assert_allclose(f[0, 20], 0.5)
    np.testing.assert_allclose(f[0, 5], 1.0 / R_)                  # positive side centroid x
    np.testing.assert_allclose(f[:, 51], 8.0 / R_ ** 3)            # mesh volume
    np.testing.assert_allclose(f[:, 53], 0.0)                      # convex: zero cost
    np.testing.assert_allclose(f[:, 54:70].sum(1), 1.0)            # histogram sums to 1
    assert np.all(f[:, R.NF:] == 0)
