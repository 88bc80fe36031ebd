"""Allocation-free Hausdorff entry point.

cuacd_hausdorff_noalloc serves callers that cannot allocate device memory
(and so cannot create a context): its scratch is a static device array, it
takes device pointers for inputs and output, and it must agree with the
allocating entry point.  Two calls in a row check that the shared static
scratch is reset between calls.  This file is named so pytest collects it
last."""
import ctypes

import numpy as np
import pytest

import cuacd_b200
from cuacd_b200 import workloads as W

pytestmark = pytest.mark.gpu
HD_ATOL = 1e-5


def _noalloc_fn():
    fn = cuacd_b200._lib.cuacd_hausdorff_noalloc
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    fn.restype = I
    fn.argtypes = [P, I, P, I, P, I, P, I, F, I, I, P, P]
    return fn


def _pairs():
    with cuacd_b200.Context(0) as ctx:
        v, t = W.hausdorff_sphere(level=4)
        (hv, ht, _), = ctx.batch_hull_dandc_mesh([v])
    a = (np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                   [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], np.float32),
         np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                   [2, 3, 7], [2, 7, 6], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]], np.int32))
    iv, it = W.icosphere(3)
    return [((hv, ht), (v, t)), (a, (iv.astype(np.float32), it))]


def test_noalloc_matches_allocating_entry():
    import torch
    fn = _noalloc_fn()
    pairs = _pairs()
    with cuacd_b200.Context(0) as ctx:
        refs = [ctx.hausdorff(*a, *b) for a, b in pairs]
    stream = torch.cuda.current_stream().cuda_stream
    for rep in range(2):                       # two calls in a row per pair
        for (a, b), ref in zip(pairs, refs):
            dav = torch.from_numpy(np.ascontiguousarray(a[0], np.float32)).cuda()
            dat = torch.from_numpy(np.ascontiguousarray(a[1], np.int32)).cuda()
            dbv = torch.from_numpy(np.ascontiguousarray(b[0], np.float32)).cuda()
            dbt = torch.from_numpy(np.ascontiguousarray(b[1], np.int32)).cuda()
            out = torch.full((1,), -1.0, dtype=torch.float32, device="cuda")
            rc = fn(dav.data_ptr(), len(a[0]), dat.data_ptr(), len(a[1]),
                    dbv.data_ptr(), len(b[0]), dbt.data_ptr(), len(b[1]),
                    2000.0, 1000, 0, out.data_ptr(), stream)
            assert rc == 0
            torch.cuda.synchronize()
            assert abs(out.item() - ref) <= HD_ATOL, (rep, out.item(), ref)


def test_noalloc_rejects_oversized_input():
    fn = _noalloc_fn()
    big = 400_000
    # sizes are checked before any pointer is touched
    rc = fn(None, 3 * big, None, big, None, 3 * big, None, big, 2000.0, 1000, 0,
            ctypes.c_void_p(1), None)
    assert rc == -2
