"""Extract the meshes of the reference's Hausdorff benchmark (the arrays of
bench/hausdorff_data.h: the bunny mesh and its hull, the 49160 mesh and its
hull) into oracle/_ref/hausdorff_bench_data.npz, so that this library can be
timed on the same inputs as the reference's benchmark binary.  The output
stays in the git-ignored oracle/_ref/.

usage:  python oracle/extract_hd_bench_data.py REFERENCE_DIR OUT.npz
"""
import re
import sys

import numpy as np


def main(ref, out):
    text = open(f"{ref}/bench/hausdorff_data.h").read()
    arrays = {}
    for m in re.finditer(r"static const (float|int) (\w+)\[\] = \{([^}]*)\};", text):
        dt = np.float32 if m.group(1) == "float" else np.int32
        arrays[m.group(2)] = np.array([float(x) if dt is np.float32 else int(x)
                                       for x in m.group(3).replace("\n", " ").split(",") if x.strip()], dt)
    rec = {}
    for name in ("BUNNY", "STL"):
        rec[f"{name}_verts"] = arrays[f"{name}_VERTS"].reshape(-1, 3)
        rec[f"{name}_tris"] = arrays[f"{name}_TRIS"].reshape(-1, 3)
        rec[f"{name}_hull_verts"] = arrays[f"{name}_HULL_VERTS"].reshape(-1, 3)
        rec[f"{name}_hull_tris"] = arrays[f"{name}_HULL_TRIS"].reshape(-1, 3)
    np.savez(out, **rec)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
