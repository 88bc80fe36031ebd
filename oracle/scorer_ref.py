"""FP64 numpy restatement of the learned candidate scorer: feature rows,
MLP forward, loss, backward and one AdamW step.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the scorer's
GPU kernels (cuacd_b200/csrc/scorer.cu).  The scorer has no counterpart in
the reference; this file restates the library's own definitions (feature
layout, 240-256-256-1 ReLU MLP, loss mean((y - 10 t)^2), AdamW with
decoupled decay on weight matrices only) so the BF16 tensor-core kernels
can be checked against exact arithmetic.
"""
import numpy as np

K, NF, H, SKETCH, TSCALE = 240, 230, 256, 80, 10.0


def unpack(p):
    p = np.asarray(p, np.float64)
    o, out = 0, {}
    for name, shape in (("W1", (K, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H,)), ("b3", (1,))):
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    assert o == len(p)
    return out


def pack(d):
    return np.concatenate([d[n].ravel() for n in ("W1", "b1", "W2", "b2", "W3", "b3")])


def forward(p, X, mean=None, inv_std=None):
    """Raw network output (T_SCALE x the predicted score) and activations;
    features are standardised first, (x - mean) * inv_std."""
    d = unpack(p)
    X = np.asarray(X, np.float64)
    if mean is not None:
        X = (X - np.asarray(mean, np.float64)) * np.asarray(inv_std, np.float64)
    Z1 = X @ d["W1"] + d["b1"]
    H1 = np.maximum(Z1, 0.0)
    Z2 = H1 @ d["W2"] + d["b2"]
    H2 = np.maximum(Z2, 0.0)
    Y = H2 @ d["W3"] + d["b3"][0]
    return Y, (X, H1, H2)


def loss_grad(p, X, T):
    """(loss, flat gradient) of loss = mean((Y - 10 T)^2)."""
    d = unpack(p)
    Y, (X, H1, H2) = forward(p, X)
    b = len(Y)
    e = Y - TSCALE * np.asarray(T, np.float64)
    loss = float(np.mean(e * e))
    dY = 2.0 * e / b
    g = {"W3": H2.T @ dY, "b3": np.array([dY.sum()])}
    dH2 = np.outer(dY, d["W3"]) * (H2 > 0)
    g["W2"] = H1.T @ dH2
    g["b2"] = dH2.sum(0)
    dH1 = (dH2 @ d["W2"].T) * (H1 > 0)
    g["W1"] = X.T @ dH1
    g["b1"] = dH1.sum(0)
    return loss, pack(g)


def adamw_step(p, g, m, v, step, lr, wd, b1=0.9, b2=0.999, eps=1e-8):
    """One AdamW update (step counts from 1); decay applies to W1, W2, W3."""
    p, g = np.asarray(p, np.float64).copy(), np.asarray(g, np.float64)
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    decay = np.zeros_like(p)
    o = 0
    for name, n, dec in (("W1", K * H, 1), ("b1", H, 0), ("W2", H * H, 1), ("b2", H, 0), ("W3", H, 1), ("b3", 1, 0)):
        decay[o:o + n] = dec
        o += n
    p -= lr * wd * p * decay
    p -= lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v


def mesh_volume(v, t):
    v = np.asarray(v, np.float64)
    a, b, c = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    return float(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0)


def part_cost_rv(hull_vol, mesh_vol):
    """Volume-difference cost of a part: 0.3 x the radius of the sphere whose
    volume is hull - mesh (cuda/la_common.cuh:21-34)."""
    diff = max(hull_vol - mesh_vol, 0.0)
    return float(0.3 * np.cbrt(3.0 / (4.0 * np.pi) * diff))


def features(verts, tris, planes, hull_vol, cost_rv=part_cost_rv):
    """Feature rows [n, 240] of planes (a, b, c, d) on one part."""
    v = np.asarray(verts, np.float64)
    nv = len(v)
    c = v.mean(0)
    r = v - c
    m2 = np.array([np.mean(r[:, 0] ** 2), np.mean(r[:, 1] ** 2), np.mean(r[:, 2] ** 2),
                   np.mean(r[:, 0] * r[:, 1]), np.mean(r[:, 0] * r[:, 2]), np.mean(r[:, 1] * r[:, 2])])
    lo, hi = r.min(0), r.max(0)
    R = 0.5 * np.linalg.norm(hi - lo)
    if not R > 0:
        R = 1.0
    mv = abs(mesh_volume(v, np.asarray(tris)))
    rv = cost_rv(float(hull_vol), mv)
    out = np.zeros((len(planes), K))
    sk = (np.arange(SKETCH) * nv) // SKETCH
    for p, pl in enumerate(np.asarray(planes, np.float64)):
        n, d = pl[:3], pl[3]
        f = out[p]
        sd = v @ n + d
        b = np.clip(np.floor((sd / R + 1.0) * 8.0), 0, 15).astype(int)
        hist = np.bincount(b, minlength=16)[:16]
        for s, sel in enumerate((sd > 0, sd < 0)):
            q = r[sel]
            cnt = len(q)
            f[4 + 16 * s] = cnt / nv
            if cnt:
                f[5 + 16 * s:8 + 16 * s] = q.mean(0) / R
                mm = [q[:, 0] ** 2, q[:, 1] ** 2, q[:, 2] ** 2, q[:, 0] * q[:, 1], q[:, 0] * q[:, 2], q[:, 1] * q[:, 2]]
                f[8 + 16 * s:14 + 16 * s] = [np.mean(x) / R ** 2 for x in mm]
                f[14 + 16 * s:17 + 16 * s] = q.min(0) / R
                f[17 + 16 * s:20 + 16 * s] = q.max(0) / R
        f[0:3] = n
        f[3] = (d + n @ c) / R
        f[36:39] = c
        f[39:45] = m2 / R ** 2
        f[45:48] = lo / R
        f[48:51] = hi / R
        f[51] = mv / R ** 3
        f[52] = hull_vol / R ** 3
        f[53] = rv / R
        f[54:70] = hist / nv
        x = r[sk]
        s_d = v[sk] @ n + d
        along = x @ n
        rad = np.sqrt(np.maximum((x * x).sum(1) - along ** 2, 0.0))
        f[70:70 + 2 * SKETCH:2] = s_d / R
        f[71:71 + 2 * SKETCH:2] = rad / R
    return out
