"""Train the learned candidate scorer on the GPU and write its weights.

    python -m cuacd_b200.train_scorer [--meshes 1500] [--epochs 60] [--out PATH]

Pairs come from the exact evaluator itself: for each seeded synthetic part
(and the two parts its best plane leaves), every candidate plane is cut,
hulled and scored exactly; the features are the library's GPU feature rows
and the target is the exact score minus its part's mean.
Training parts use a wide plane set (up to 64 concave-edge planes and 14
axis cuts); validation and held-out parts use one search level's 30 planes
(27 concave-edge + 3 axis midpoints).  Training runs the library's BF16
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
    ap.add_argument("--out", default=S.WEIGHTS_PATH)
    a = ap.parse_args()

    ctx = cuacd_b200.Context(0)
    sc = S.Scorer(ctx, seed=a.seed)
    t0 = time.perf_counter()
    X, T, G = S.build_dataset(ctx, sc, S.training_meshes(a.meshes, a.seed), plane_set=WIDE)
    Xv, Tv, Gv = S.build_dataset(ctx, sc, S.training_meshes(a.val, a.seed + 500))
    Xh, Th, Gh = S.build_dataset(ctx, sc, S.training_meshes(a.holdout, a.seed + 1000))
    t_data = time.perf_counter() - t0
    sc.fit_normalizer(X)
    Tc = S.centered(T, G)
    before = S.ranking_quality(sc.predict(Xh), Th, Gh)
    t0 = time.perf_counter()
    best = (np.inf, None, 0)
    history = []
    for c in range(a.epochs // a.chunk):
        lr = a.lr * 0.5 * (1 + np.cos(np.pi * c / (a.epochs // a.chunk)))    # cosine decay per chunk
        mse = sc.train(X, Tc, epochs=a.chunk, batch=a.batch, lr=lr, wd=a.wd, seed=a.seed + c)
        hit, reg, _ = S.ranking_quality(sc.predict(Xv), Tv, Gv)
        history.append((round(mse, 6), round(hit, 3), round(reg, 5)))
        if reg < best[0]:
            best = (reg, sc.params(), (c + 1) * a.chunk)
    sc.set_params(best[1])
    t_train = time.perf_counter() - t0
    ph = sc.predict(Xh)
    hit, reg, rreg = S.ranking_quality(ph, Th, Gh)
    sizes = np.bincount(Gh)
    info = {
        "pairs": int(len(T)), "parts": int(G.max() + 1), "val_pairs": int(len(Tv)),
        "holdout_pairs": int(len(Th)), "holdout_parts": int(Gh.max() + 1),
        "holdout_planes_per_part": float(sizes.mean()), "data_s": round(t_data, 1), "train_s": round(t_train, 1),
        "epochs_kept": best[2], "history": history, "holdout_mse": float(np.mean((ph - S.centered(Th, Gh)) ** 2)),
        "holdout_top8_hit": hit, "random_top8_hit": float(np.mean(np.minimum(8, sizes) / sizes)),
        "holdout_top8_regret": reg, "random_top8_regret": rreg, "untrained_top8": before,
        "batch": a.batch, "lr": a.lr, "wd": a.wd,
    }
    sc.save(a.out, info=json.dumps(info))
    print(json.dumps(info))


if __name__ == "__main__":
    main()
