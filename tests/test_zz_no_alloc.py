"""xmpIntegersPowmNoAlloc against the regular xmpIntegersPowm and GMP, through the C ABI.

The allocation-free entry point serves callers that cannot allocate device
memory (a latency-critical path where cudaMalloc would synchronise the
device, or an allocator that only hands out the operand buffers): it keeps
its window tables in a fixed device array shared by every call.  These tests
allocate the operand buffers themselves (the caller's job), run two different
batches in a row through the new entry point and require bit-identical
results to the existing entry point and to GMP for both, so the second call
cannot be reading stale tables from the first; they also check the documented
size limit, a batch large enough that the window must shrink to fit the
array, and an output that aliases an input.  Kept in their own file, collected
last, and independent of the other tests' state.
"""
import ctypes

import numpy as np
import pytest

import oracle
import xmp_b200 as xmp

pytestmark = pytest.mark.gpu


def _interleave(rows, stride):
    """Compact rows (count x nlimbs) -> the library's device layout (limb j of
    instance i at ((j/4)*stride + i)*4 + j%4), as a flat uint32 array."""
    count, n = rows.shape
    g = (n + 3) // 4
    out = np.zeros((g, stride, 4), dtype=np.uint32)
    padded = np.zeros((count, g * 4), dtype=np.uint32)
    padded[:, :n] = rows
    out[:, :count, :] = padded.reshape(count, g, 4).transpose(1, 0, 2)
    return out.reshape(-1)


def _deinterleave(flat, count, n, stride):
    g = (n + 3) // 4
    return flat.reshape(g, stride, 4).transpose(1, 0, 2).reshape(stride, g * 4)[:count, :n].copy()


def _regular_powm(h, x, e, m, bits, ebits):
    count = len(m)
    X, E, M, O = h.integers(bits, count, x), h.integers(ebits, count, e), h.integers(bits, count, m), \
        h.integers(bits, count)
    xmp.powm(h, O, X, E, M, count)
    got = O.export()
    for v in (X, E, M, O):
        v.destroy()
    return got


def test_powm_no_alloc_matches_regular_entry_point_twice():
    import torch

    torch.cuda.set_device(0)
    lib = xmp.lib()
    h = xmp.Handle()
    bits, ebits, count = 2048, 2048, 500
    n, en = bits // 32, ebits // 32
    stride = 512
    stream = torch.cuda.current_stream()
    try:
        for call, seed in enumerate((71, 72)):  # two calls in a row, different inputs
            m = oracle.full_length_odd(seed, count, n)
            x = oracle.below(seed + 1, m)
            e = oracle.random_limbs(seed + 2, count, en)
            want = _regular_powm(h, x, e, m, bits, ebits)
            dx, de, dm = (torch.from_numpy(_interleave(v, stride).view(np.int32)).cuda() for v in (x, e, m))
            dout = torch.zeros_like(dx)
            rc = lib.xmpIntegersPowmNoAlloc(stream.cuda_stream, dout.data_ptr(), dx.data_ptr(), de.data_ptr(),
                                            dm.data_ptr(), bits, ebits, stride, count)
            assert rc == 0, xmp.XmpError(rc).name
            torch.cuda.synchronize()
            got = _deinterleave(dout.cpu().numpy().view(np.uint32), count, n, stride)
            assert np.array_equal(got, want), "call %d differs from xmpIntegersPowm" % (call + 1)
            gmp, _ = oracle.powm(x, e, m, count)
            assert np.array_equal(got, gmp), "call %d differs from GMP" % (call + 1)
        # sizes beyond the fixed scratch are rejected, nothing is launched
        big = 1 << 16
        rc = lib.xmpIntegersPowmNoAlloc(stream.cuda_stream, dout.data_ptr(), dx.data_ptr(), de.data_ptr(),
                                        dm.data_ptr(), 4096, 4096, big, big)
        assert rc == xmp.ERR["xmpErrorIncreaseScratchLimit"]
        rc = lib.xmpIntegersPowmNoAlloc(stream.cuda_stream, dout.data_ptr(), dx.data_ptr(), de.data_ptr(),
                                        dm.data_ptr(), bits, ebits, count - 1, count)
        assert rc == xmp.ERR["xmpErrorInvalidCount"]
    finally:
        h.destroy()


def _no_alloc(lib, stream, out, x, e, m, bits, ebits, stride, count):
    rc = lib.xmpIntegersPowmNoAlloc(stream.cuda_stream, out.data_ptr(), x.data_ptr(), e.data_ptr(), m.data_ptr(),
                                    bits, ebits, stride, count)
    assert rc == 0, xmp.XmpError(rc).name
    torch_sync()


def torch_sync():
    import torch
    torch.cuda.synchronize()


def test_powm_no_alloc_window_shrink_and_aliasing():
    """4096-bit batch whose default-window tables exceed the 16 MiB array (the window shrinks), then the
    output written over the exponent and over the base buffers."""
    import torch

    torch.cuda.set_device(0)
    lib = xmp.lib()
    stream = torch.cuda.current_stream()
    bits, count = 4096, 640
    n, stride = bits // 32, 640
    m = oracle.full_length_odd(81, count, n)
    x = oracle.below(82, m)
    e = oracle.random_limbs(83, count, n)
    want, _ = oracle.powm(x, e, m, count)
    dx, de, dm = (torch.from_numpy(_interleave(v, stride).view(np.int32)).cuda() for v in (x, e, m))
    dout = torch.zeros_like(dx)
    _no_alloc(lib, stream, dout, dx, de, dm, bits, bits, stride, count)
    assert np.array_equal(_deinterleave(dout.cpu().numpy().view(np.uint32), count, n, stride), want)
    # out == exp
    _no_alloc(lib, stream, de, dx, de, dm, bits, bits, stride, count)
    assert np.array_equal(_deinterleave(de.cpu().numpy().view(np.uint32), count, n, stride), want)
    # out == base (2048 bits, a second shape through the same array)
    bits, count = 2048, 300
    n, stride = bits // 32, 320
    m = oracle.full_length_odd(84, count, n)
    x = oracle.below(85, m)
    e = oracle.random_limbs(86, count, n)
    want, _ = oracle.powm(x, e, m, count)
    dx, de, dm = (torch.from_numpy(_interleave(v, stride).view(np.int32)).cuda() for v in (x, e, m))
    _no_alloc(lib, stream, dx, dx, de, dm, bits, bits, stride, count)
    assert np.array_equal(_deinterleave(dx.cpu().numpy().view(np.uint32), count, n, stride), want)
