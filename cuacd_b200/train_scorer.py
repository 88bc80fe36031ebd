"""Train the learned candidate scorer on the GPU and write its weights.

    python -m cuacd_b200.train_scorer [--meshes 1500] [--epochs 60] [--out PATH]

Pairs come from the exact evaluator itself: for each seeded synthetic part
(and the two parts its best plane leaves), every candidate plane is cut,
hulled and scored exactly; the features are the library's GPU feature rows
and the target is the exact score minus its part's mean.
Training parts use a wide plane set (up to 64 concave-edge planes and 14
axis cuts); validation and held-out parts use one search level's 30 planes
(27 concave-edge + 3 axis midpoints).  With --target rv the pairs are the
search's level-0 planes at its defaults (up to 128 concave-edge planes and 30
axis cuts) scored by score_rv, the cost the search ranks by.  Training runs the library's BF16
tensor-core forward/backward and AdamW kernels; the epoch count is chosen
on the validation parts (lowest top-8 regret), and the held-out parts
(other seeds) report how often the top-8 predictions contain the exact best
plane, against random choice.
"""
import argparse
import json
import time

import numpy as np

import cuacd_b200
from cuacd_b200 import scorer as S

WIDE = {"n_concave_edges": 16, "width": 14, "max_concave": 64}
# the search's level-0 set at its defaults (32 sampled concave edges, width 30)
SEARCH = {"n_concave_edges": 32, "width": 30, "max_concave": 128}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--meshes", type=int, default=1500)
    ap.add_argument("--val", type=int, default=120)
    ap.add_argument("--holdout", type=int, default=120)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--chunk", type=int, default=5)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--wd", type=float, default=1e-2)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--out", default=None)
    ap.add_argument("--target", default="full", choices=["full", "rv", "path"],
                    help="full: score_full of one level's 30 planes (the evaluator); "
                         "rv: score_rv of the search's level-0 planes; "
                         "path: the search's own path cost of each level-0 plane (the lookahead)")
    ap.add_argument("--iters", type=int, default=12, help="path target: search iterations traced per mesh")
    ap.add_argument("--topk", type=int, default=8)
    a = ap.parse_args()
    if a.out is None:
        a.out = {"full": S.WEIGHTS_PATH, "rv": S.RV_WEIGHTS_PATH, "path": S.PATH_WEIGHTS_PATH}[a.target]
    if a.target == "path":
        return train_path(a)
    train_set = WIDE if a.target == "full" else SEARCH
    eval_set = None if a.target == "full" else SEARCH

    ctx = cuacd_b200.Context(0)
    sc = S.Scorer(ctx, seed=a.seed)
    t0 = time.perf_counter()
    X, T, G = S.build_dataset(ctx, sc, S.training_meshes(a.meshes, a.seed), plane_set=train_set, target=a.target)
    Xv, Tv, Gv = S.build_dataset(ctx, sc, S.training_meshes(a.val, a.seed + 500), plane_set=eval_set, target=a.target)
    Xh, Th, Gh = S.build_dataset(ctx, sc, S.training_meshes(a.holdout, a.seed + 1000), plane_set=eval_set,
                                 target=a.target)
    t_data = time.perf_counter() - t0
    sc.fit_normalizer(X)
    Tc = S.centered(T, G)
    before = S.ranking_quality(sc.predict(Xh), Th, Gh, k=a.topk)
    t0 = time.perf_counter()
    best = (np.inf, None, 0)
    history = []
    for c in range(a.epochs // a.chunk):
        lr = a.lr * 0.5 * (1 + np.cos(np.pi * c / (a.epochs // a.chunk)))    # cosine decay per chunk
        mse = sc.train(X, Tc, epochs=a.chunk, batch=a.batch, lr=lr, wd=a.wd, seed=a.seed + c)
        hit, reg, _ = S.ranking_quality(sc.predict(Xv), Tv, Gv, k=a.topk)
        history.append((round(mse, 6), round(hit, 3), round(reg, 5)))
        if reg < best[0]:
            best = (reg, sc.params(), (c + 1) * a.chunk)
    sc.set_params(best[1])
    t_train = time.perf_counter() - t0
    ph = sc.predict(Xh)
    hit, reg, rreg = S.ranking_quality(ph, Th, Gh, k=a.topk)
    sizes = np.bincount(Gh)
    info = {
        "pairs": int(len(T)), "parts": int(G.max() + 1), "val_pairs": int(len(Tv)),
        "holdout_pairs": int(len(Th)), "holdout_parts": int(Gh.max() + 1),
        "holdout_planes_per_part": float(sizes.mean()), "data_s": round(t_data, 1), "train_s": round(t_train, 1),
        "epochs_kept": best[2], "history": history, "holdout_mse": float(np.mean((ph - S.centered(Th, Gh)) ** 2)),
        "target": a.target, "topk": a.topk,
        "holdout_topk_hit": hit, "random_topk_hit": float(np.mean(np.minimum(a.topk, sizes) / sizes)),
        "holdout_topk_regret": reg, "random_topk_regret": rreg, "untrained_topk": before,
        "batch": a.batch, "lr": a.lr, "wd": a.wd,
    }
    sc.save(a.out, info=json.dumps(info))
    print(json.dumps(info))


def trace_set(ctx, sc, meshes, iters):
    """Rows of every traced search: features, path cost, part group."""
    Xs, Ts, Gs = [], [], []
    g0 = 0
    for v, t in meshes:
        X, c0, cb, key, _ = S.lookahead_trace(ctx, sc, v, t, max_iters=iters)
        if len(X) == 0:
            continue
        _, gid = np.unique(key, return_inverse=True)
        Xs.append(X); Ts.append(cb); Gs.append(gid + g0)
        g0 += gid.max() + 1
    return np.concatenate(Xs), np.concatenate(Ts), np.concatenate(Gs).astype(np.int64)


def train_path(a):
    """Scorer for the search's level 0: target = the path cost the exact
    search gives each level-0 plane (its best two-level mean), centred per
    cutting part, from traces of the exact search on seeded parts."""
    ctx = cuacd_b200.Context(0)
    sc = S.Scorer(ctx, seed=a.seed)
    t0 = time.perf_counter()
    X, T, G = trace_set(ctx, sc, S.training_meshes(a.meshes, a.seed), a.iters)
    Xv, Tv, Gv = trace_set(ctx, sc, S.training_meshes(a.val, a.seed + 500), a.iters)
    Xh, Th, Gh = trace_set(ctx, sc, S.training_meshes(a.holdout, a.seed + 1000), a.iters)
    t_data = time.perf_counter() - t0
    sc.fit_normalizer(X)
    Tc = S.centered(T, G)
    t0 = time.perf_counter()
    best = (np.inf, None, 0)
    history = []
    for c in range(a.epochs // a.chunk):
        lr = a.lr * 0.5 * (1 + np.cos(np.pi * c / (a.epochs // a.chunk)))
        mse = sc.train(X, Tc, epochs=a.chunk, batch=a.batch, lr=lr, wd=a.wd, seed=a.seed + c)
        hit, reg, _ = S.ranking_quality(sc.predict(Xv), Tv, Gv, k=a.topk)
        history.append((round(mse, 7), round(hit, 3), round(reg, 6)))
        if reg < best[0]:
            best = (reg, sc.params(), (c + 1) * a.chunk)
    sc.set_params(best[1])
    t_train = time.perf_counter() - t0
    ph = sc.predict(Xh)
    hit, reg, rreg = S.ranking_quality(ph, Th, Gh, k=a.topk)
    sizes = np.bincount(Gh)
    info = {"target": "path", "topk": a.topk, "rows": int(len(T)), "groups": int(G.max() + 1),
            "holdout_rows": int(len(Th)), "holdout_groups": int(Gh.max() + 1),
            "holdout_planes_per_group": float(sizes.mean()), "data_s": round(t_data, 1),
            "train_s": round(t_train, 1), "epochs_kept": best[2], "history": history,
            "holdout_topk_hit": hit, "random_topk_hit": float(np.mean(np.minimum(a.topk, sizes) / sizes)),
            "holdout_topk_regret": reg, "random_topk_regret": rreg, "iters": a.iters}
    sc.save(a.out, info=json.dumps(info))
    print(json.dumps(info))


if __name__ == "__main__":
    main()
