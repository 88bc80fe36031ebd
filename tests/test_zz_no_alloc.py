"""Allocation-free Hausdorff entry point.

cuacd_hausdorff_noalloc serves callers that cannot allocate device memory
(and so cannot create a context): its scratch is a static device array, it
takes device pointers for inputs and output, and it must agree with the
allocating entry point and with the oracle.  Two calls in a row check that
the shared static scratch is reset between calls; the device's free memory
before and after repeated calls checks that nothing is allocated.  This file
is named so pytest collects it last."""
import ctypes

import numpy as np
import pytest

import cuacd_b200
from cuacd_b200 import workloads as W

pytestmark = pytest.mark.gpu
HD_ATOL = 1e-5
TOO_LARGE, BAD_ARGS = -2, -3


def _noalloc_fn():
    fn = cuacd_b200._lib.cuacd_hausdorff_noalloc
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    fn.restype = I
    fn.argtypes = [P, I, P, I, P, I, P, I, F, I, I, P, P]
    return fn


def _cube():
    return (np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                      [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], np.float32),
            np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                      [2, 3, 7], [2, 7, 6], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]], np.int32))


def _pairs():
    with cuacd_b200.Context(0) as ctx:
        v, t = W.hausdorff_sphere(level=4)
        (hv, ht, _), = ctx.batch_hull_dandc_mesh([v])
    iv, it = W.icosphere(3)
    return [((hv, ht), (v, t)), (_cube(), (iv.astype(np.float32), it))]


def _dev(a, dtype, pad_rows=0):
    import torch
    a = np.ascontiguousarray(a, dtype).reshape(-1, 3)
    if pad_rows:
        a = np.concatenate([a, np.zeros((pad_rows, 3), dtype)])
    return torch.from_numpy(a).cuda()


def _call(fn, a, b, out, stream, a_nv=None):
    (dav, dat), (dbv, dbt) = a, b
    return fn(dav.data_ptr(), len(dav) if a_nv is None else a_nv, dat.data_ptr(), len(dat),
              dbv.data_ptr(), len(dbv), dbt.data_ptr(), len(dbt),
              2000.0, 1000, 0, out.data_ptr(), stream)


def test_noalloc_matches_allocating_entry_and_oracle():
    import torch
    from oracle import oracle as O
    fn = _noalloc_fn()
    pairs = _pairs()
    with cuacd_b200.Context(0) as ctx:
        refs = [ctx.hausdorff(*a, *b) for a, b in pairs]
    orc = [O.hausdorff(*a, *b, threads=8) for a, b in pairs]
    for r, o in zip(refs, orc):
        assert abs(r - o) <= HD_ATOL, (r, o)
    dev = [((_dev(a[0], np.float32), _dev(a[1], np.int32)), (_dev(b[0], np.float32), _dev(b[1], np.int32)))
           for a, b in pairs]
    outs = [torch.full((1,), -1.0, dtype=torch.float32, device="cuda") for _ in range(2 * len(pairs))]
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free0 = None
    for rep in range(2):                       # two calls in a row per pair
        for i, ((a, b), ref, o) in enumerate(zip(dev, refs, orc)):
            out = outs[rep * len(pairs) + i]
            assert _call(fn, a, b, out, stream) == 0
            torch.cuda.synchronize()
            assert abs(out.item() - ref) <= HD_ATOL, (rep, out.item(), ref)
            assert abs(out.item() - o) <= HD_ATOL, (rep, out.item(), o)
            if free0 is None:                  # after the first call (symbol set-up done)
                free0 = torch.cuda.mem_get_info()[0]
    assert torch.cuda.mem_get_info()[0] == free0, "the entry point allocated device memory"


def test_noalloc_empty_surface_matches_allocating_entry():
    import torch
    fn = _noalloc_fn()
    cv, ct = _cube()
    ev, et = np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32)
    with cuacd_b200.Context(0) as ctx:
        ref = ctx.hausdorff(ev, et, cv, ct)
    a = (_dev(cv, np.float32, pad_rows=1)[:0], _dev(ct, np.int32, pad_rows=1)[:0])
    b = (_dev(cv, np.float32), _dev(ct, np.int32))
    out = torch.full((1,), -1.0, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        assert _call(fn, a, b, out, stream) == 0
        torch.cuda.synchronize()
        assert out.item() == ref, (out.item(), ref)


def test_noalloc_out_of_range_index_gives_nan():
    # The vertex buffer keeps one spare row beyond the count passed, so the
    # bad index (== nv) would still land inside the allocation; the
    # device-side scan must refuse it before any kernel reads through it.
    import torch
    fn = _noalloc_fn()
    cv, ct = _cube()
    bad_t = ct.copy()
    bad_t[5, 1] = len(cv)
    a = (_dev(cv, np.float32, pad_rows=1), _dev(bad_t, np.int32))
    b = (_dev(cv, np.float32), _dev(ct, np.int32))
    out = torch.full((1,), -1.0, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert _call(fn, a, b, out, stream, a_nv=len(cv)) == 0
    torch.cuda.synchronize()
    assert np.isnan(out.item())
    # the next good call on the same static block is unaffected
    with cuacd_b200.Context(0) as ctx:
        ref = ctx.hausdorff(cv, ct, cv, ct)
    good = (_dev(cv, np.float32), _dev(ct, np.int32))
    assert _call(fn, good, b, out, stream) == 0
    torch.cuda.synchronize()
    assert abs(out.item() - ref) <= HD_ATOL, (out.item(), ref)


def test_noalloc_rejects_bad_sizes():
    fn = _noalloc_fn()
    # sizes are checked before any pointer is touched
    big = 400_000
    assert fn(None, 3 * big, None, big, None, 3 * big, None, big, 2000.0, 1000, 0,
              ctypes.c_void_p(1), None) == TOO_LARGE
    imax = 2**31 - 1
    assert fn(None, imax, None, imax, None, 3, None, 1, 2000.0, 1000, 0,
              ctypes.c_void_p(1), None) == TOO_LARGE
    assert fn(None, 3, None, 1, None, imax, None, imax, 2000.0, 1000, 0,
              ctypes.c_void_p(1), None) == TOO_LARGE
    assert fn(None, -1, None, 1, None, 3, None, 1, 2000.0, 1000, 0,
              ctypes.c_void_p(1), None) == BAD_ARGS
    assert fn(None, 3, None, 1, None, 3, None, -5, 2000.0, 1000, 0,
              ctypes.c_void_p(1), None) == BAD_ARGS
    assert fn(None, 3, None, 1, None, 3, None, 1, 2000.0, 1000, 0, None, None) == BAD_ARGS
