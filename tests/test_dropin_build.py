"""The drop-in boundary from the reference's side, on the CPU: the
reference's CPython module (csrc/module.c, unmodified) compiles against
include/ (cuacd_b200.h plus the reference header names that forward to it)
and links against libcuacd_b200.so alone -- gpu_preprocess included -- and
the module it makes imports with the reference's full method table."""
import importlib.machinery
import importlib.util
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
METHODS = {"init", "destroy", "set_fatbin", "pool_usage", "heap_stats", "heap_compact", "test_warp_sort",
           "hull_dandc", "test_mesh_volume", "batch_mesh_volume", "test_plane_cut", "test_postprocess_dc",
           "lookahead_decompose", "kdop_hull", "test_hausdorff", "mesh_audit", "preprocess"}


def _import(path):
    loader = importlib.machinery.ExtensionFileLoader("_gpu", path)
    mod = importlib.util.module_from_spec(importlib.util.spec_from_loader("_gpu", loader))
    loader.exec_module(mod)
    return mod


def test_reference_module_builds_and_links(tmp_path):
    from oracle import oracle as O
    ref = O.reference_tree()
    if ref is None:
        pytest.skip("the reference tree is not on this machine")
    out = tmp_path / "_gpu_dropin.so"
    r = subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile.ref"), f"REF={ref}",
                        f"OUT={tmp_path}", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    undefined = subprocess.run(["nm", "-D", "--undefined-only", str(out)], capture_output=True, text=True).stdout
    needed = {ln.split()[-1] for ln in undefined.splitlines() if ln.split() and ln.split()[-1].startswith("gpu_")}
    exported = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "cuacd_b200", "libcuacd_b200.so")],
                              capture_output=True, text=True).stdout
    have = {ln.split()[-1] for ln in exported.splitlines() if ln.split()}
    assert needed and needed <= have, needed - have
    assert "lookahead_decompose" in have


def test_built_module_method_table():
    path = os.path.join(ROOT, "oracle", "_ref", "_gpu_dropin.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref/_gpu_dropin.so not built")
    mod = _import(path)
    assert METHODS <= set(dir(mod)), METHODS - set(dir(mod))
