"""Build recipe for libcuacd_b200.so (nvcc, sm_100a only).

Each .cu under csrc/ is one translation unit with its own kernels; they are
compiled in parallel and linked into one shared library next to this file.
No fast-math: several device expressions must round exactly as written
(IEEE division and square root, explicit fmaf) so integer results match the
checker bit for bit.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcuacd_b200.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


# Per-file flags: the FP32/FP64 expressions of the cut, the plane generator,
# the audit's zero-area test and the remesh must not be contracted.
PER_FILE = {"cut.cu": ["-fmad=false"], "concave.cu": ["-fmad=false"], "audit.cu": ["-fmad=false"],
            "remesh.cu": ["-fmad=false"]}


def _compile(src, extra):
    obj = os.path.join(BUILD, src[:-3] + ".o")
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "cuacd_b200.h")]
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj, ""
    cmd = [NVCC, *ARCH, *FLAGS, *PER_FILE.get(src, []), *extra, "-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    srcs = sources()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, extra), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log, file=sys.stderr)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
    print(LIB)
