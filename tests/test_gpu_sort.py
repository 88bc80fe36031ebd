"""gpu_test_warp_sort: exact (y,x,z,index) order (reference
tests/test_warp_sort.py:13-17 oracle is np.lexsort)."""
import ctypes

import numpy as np
import pytest

import cuacd_b200

pytestmark = pytest.mark.gpu


def _sort(ctx, arrays):
    off = np.zeros(len(arrays) + 1, np.int32)
    for i, a in enumerate(arrays):
        off[i + 1] = off[i] + len(a)
    packed = np.ascontiguousarray(np.concatenate(arrays).astype(np.int32))
    fn = cuacd_b200._fn("gpu_test_warp_sort")
    rc = fn(ctx.handle, ctypes.c_void_p(packed.ctypes.data), int(off[-1]), ctypes.c_void_p(off.ctypes.data), len(arrays))
    assert rc == 0
    return [packed[off[i]:off[i + 1]] for i in range(len(arrays))]


def test_orders(ctx):
    rng = np.random.default_rng(0)
    arrays = []
    for n in (1, 2, 31, 32, 33, 1000, 5000, 20000):
        a = np.c_[rng.integers(-50, 50, (n, 3)), np.arange(n)].astype(np.int32)
        arrays.append(a)
    arrays.append(np.c_[np.zeros((64, 3), int), np.arange(64)[::-1]].astype(np.int32))   # all equal keys
    sorted_ = _sort(ctx, [a.copy() for a in arrays])
    for a, s in zip(arrays, sorted_):
        ref = a[np.lexsort((a[:, 3], a[:, 2], a[:, 0], a[:, 1]))]
        np.testing.assert_array_equal(s, ref)
