"""The C-ABI library loads and exports every symbol that include/cuacd_b200.h
(the drop-in ABI) and include/cuacd_b200_diag.h (diagnostics) declare (CPU
only; no compute call needs a GPU here)."""
import ctypes
import os
import re

from conftest import ROOT


def declared_functions():
    src = "".join(open(os.path.join(ROOT, "include", h)).read() for h in ("cuacd_b200.h", "cuacd_b200_diag.h"))
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b([a-z_][a-z0-9_]*)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "sizeof")))


def test_library_exports_all_declared_symbols():
    import cuacd_b200
    lib = ctypes.CDLL(cuacd_b200.native_library_path())
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_package_fails_loudly_without_library(tmp_path):
    """Importing from a copy without the .so raises ImportError (no fallback)."""
    import shutil, subprocess, sys
    pkg = tmp_path / "cuacd_b200"
    shutil.copytree(os.path.join(ROOT, "cuacd_b200"), pkg,
                    ignore=shutil.ignore_patterns("*.so", "_build", "__pycache__"))
    r = subprocess.run([sys.executable, "-c", "import cuacd_b200"], cwd=tmp_path,
                       capture_output=True, text=True)
    assert r.returncode != 0 and "native library is missing" in r.stderr
