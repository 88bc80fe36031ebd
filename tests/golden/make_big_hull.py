"""Generate tests/golden/hull_big.npz: hulls with more than 65,536 vertices,
computed by the oracle (minutes of CPU; the GPU tests only compare).

  ico7_idx     input indices of the exact hull vertices of the 163,842
               vertices of a level-7 icosphere (79,206 on the hull grid)
  cut_plane    a plane leaving 95 % of that sphere on its positive side
  cut_*        the oracle's candidate evaluation of the level-7 sphere mesh
               on that plane (no Hausdorff): fragment and hull sizes, volumes

usage: python tests/golden/make_big_hull.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from cuacd_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

PLANE = np.array([[1.0, 0.0, 0.0, 0.9]], np.float32)


def main():
    v, t = W.icosphere(7)
    v = v.astype(np.float32)
    idx = O.hull(v)[0]
    r = O.eval_candidates(v, t, PLANE, hausdorff=False, threads=os.cpu_count() or 1)[0]
    np.savez_compressed(os.path.join(HERE, "hull_big.npz"), ico7_idx=np.asarray(idx, np.int32), cut_plane=PLANE,
                        cut_ok=np.int32(r["ok"]), cut_nv=np.array(r["nv"], np.int32),
                        cut_nt=np.array(r["nt"], np.int32), cut_hull_nv=np.array(r["hull_nv"], np.int32),
                        cut_hull_nt=np.array(r["hull_nt"], np.int32), cut_hull_vol=np.array(r["hull_vol"]),
                        cut_mesh_vol=np.array(r["mesh_vol"]))
    print(len(idx), r["nv"], r["hull_nv"])


if __name__ == "__main__":
    main()
