"""Device allocations go through the handle's allocator callbacks
(xmpHandleCreateWithMemoryFunctions, reference src/xmp.cu:43-65); an
allocator that refuses gives xmpErrorInvalidCudaMalloc, the handle stays
usable, and a handle whose allocator refuses from the start is still
created (it falls back from the compiled-in selector to the heuristic)."""
import ctypes

import numpy as np
import pytest
import torch

import oracle
import xmp_b200 as xmp

pytestmark = pytest.mark.gpu

ALLOC = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_size_t)
FREE = ctypes.CFUNCTYPE(None, ctypes.c_void_p)
INVALID_CUDA_MALLOC = 4


class Allocator:
    def __init__(self):
        self.fail = False
        self.calls = 0
        self.live = {}

        @ALLOC
        def alloc(n):
            self.calls += 1
            if self.fail:
                return None
            p = torch.cuda.caching_allocator_alloc(max(int(n), 1))
            self.live[p] = n
            return p

        @FREE
        def free(p):
            if p and p in self.live:
                del self.live[p]
                torch.cuda.caching_allocator_delete(p)

        self.alloc, self.free = alloc, free

    def handle(self):
        h = ctypes.c_void_p()
        xmp.check(xmp.lib().xmpHandleCreateWithMemoryFunctions(
            ctypes.byref(h), None, None, ctypes.cast(self.alloc, ctypes.c_void_p),
            ctypes.cast(self.free, ctypes.c_void_p)))
        return h


def test_allocator_used_and_refusal_reported():
    torch.cuda.init()
    A = Allocator()
    h = A.handle()
    L = xmp.lib()
    try:
        x, y, o = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        n0 = A.calls
        xmp.check(L.xmpIntegersCreate(h, ctypes.byref(x), 1024, 64))
        assert A.calls > n0 and A.live  # the integers came from the caller's allocator
        A.fail = True
        assert L.xmpIntegersCreate(h, ctypes.byref(y), 1024, 64) == INVALID_CUDA_MALLOC
        A.fail = False
        # the handle still works: a powm through it is exact
        m = oracle.full_length_odd(3, 64, 32)
        b = oracle.below(4, m)
        e = oracle.random_limbs(5, 64, 32)
        for arr in (y, o):
            xmp.check(L.xmpIntegersCreate(h, ctypes.byref(arr), 1024, 64))
        X = ctypes.c_void_p()
        xmp.check(L.xmpIntegersCreate(h, ctypes.byref(X), 1024, 64))
        for arr, rows in ((x, b), (y, e), (X, m)):
            xmp.check(L.xmpIntegersImport(h, arr, 32, -1, 4, 0, 0, rows.ctypes.data, 64))
        xmp.check(L.xmpIntegersPowm(h, o, x, y, X, 64))
        out = np.zeros((64, 32), dtype=np.uint32)
        w = ctypes.c_uint32()
        xmp.check(L.xmpIntegersExport(h, out.ctypes.data, ctypes.byref(w), -1, 4, 0, 0, o, 64))
        want, _ = oracle.powm(b, e, m, 64)
        assert np.array_equal(out, want)
        for arr in (x, y, o, X):
            xmp.check(L.xmpIntegersDestroy(h, arr))
    finally:
        xmp.check(L.xmpHandleDestroy(h))
    assert not A.live  # everything handed out was given back


def test_handle_with_refusing_allocator():
    A = Allocator()
    A.fail = True
    h = A.handle()  # created all the same: the selector table could not be built, the heuristic is used
    try:
        x = ctypes.c_void_p()
        assert xmp.lib().xmpIntegersCreate(h, ctypes.byref(x), 256, 8) == INVALID_CUDA_MALLOC
    finally:
        xmp.check(xmp.lib().xmpHandleDestroy(h))
