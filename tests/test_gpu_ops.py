"""CUDA elementwise / mul / divmod / import-export / error paths vs the oracle.

Mirrors the reference's unit-test pattern (unit_tests/test.cu): seeded random
data, shuffled index policies, broadcast counts (M = 100 and 1), odd
precisions and in-place variants, compared limb by limb with the GMP oracle.
"""
import numpy as np
import pytest

import oracle
import xmp_b200 as xmp
from tests.helpers import ints_from_rows, rows_from_ints

pytestmark = pytest.mark.gpu

N, M = 2000, 100


def _rows(seed, count, bits):
    return oracle.random_limbs(seed, count, bits // 32)


def _perm(seed, n):
    return np.random.default_rng(seed).permutation(n).astype(np.uint32)


BIN = {"add": xmp.add, "sub": xmp.sub, "and": xmp.and_, "ior": xmp.ior, "xor": xmp.xor, "mul": xmp.mul,
       "div": xmp.div, "mod": xmp.mod}

# (out bits, a bits, b bits, a count, b count)
GRID = [(64, 32, 32, N, N), (288, 256, 256, N, N), (288, 256, 256, N, M), (544, 512, 512, N, 1),
        (192, 160, 160, N, N), (384, 384, 384, N, N), (1056, 1024, 1024, N, N), (8224, 8192, 8192, 64, 64),
        (256, 256, 128, N, N), (352, 352, 352, M, N)]


@pytest.mark.parametrize("op", ["add", "sub", "and", "ior", "xor", "mul"])
@pytest.mark.parametrize("shape", GRID)
def test_binary_indexed(handle, op, shape):
    bo, ba, bb, na, nb = shape
    if op == "mul":
        bo = max(ba, bb) * 2 if ba + bb <= 4096 else max(ba, bb)
    count = min(N, max(na, nb))
    a, b = _rows(1, na, ba), _rows(2, nb, bb)
    oi, ai, bi = _perm(3, count), _perm(4, na), _perm(5, nb)
    want = oracle.binary(op, a, b, bo // 32, count, out_index=oi, a_index=ai, b_index=bi)
    A, B, C = handle.integers(ba, na, a), handle.integers(bb, nb, b), handle.integers(bo, count)
    pol = handle.policy()
    pol.set_indices(0, oi)
    pol.set_indices(1, ai)
    pol.set_indices(2, bi)
    handle.set_policy(pol)
    try:
        BIN[op](handle, C, A, B, count)
    finally:
        handle.set_policy(None)
    got = C.export()
    assert np.array_equal(got, want), (op, shape)
    # no indices
    want2 = oracle.binary(op, a, b, bo // 32, count)
    BIN[op](handle, C, A, B, count)
    assert np.array_equal(C.export(), want2), (op, shape, "plain")
    for x in (A, B, C):
        x.destroy()
    pol.destroy()


@pytest.mark.parametrize("op", ["add", "sub", "xor", "mul"])
def test_binary_in_place(handle, op):
    bits = 256
    a, b = _rows(6, N, bits), _rows(7, N, bits)
    A, B = handle.integers(bits, N, a), handle.integers(bits, N, b)
    want = oracle.binary(op, a, b, bits // 32, N)
    BIN[op](handle, A, A, B, N)
    assert np.array_equal(A.export(), want)
    # in place with a shuffled output index: staged through the temporary output
    A.import_(a)
    oi = _perm(8, N)
    want = oracle.binary(op, a, b, bits // 32, N, out_index=oi, init=a)
    pol = handle.policy()
    pol.set_indices(0, oi)
    handle.set_policy(pol)
    try:
        BIN[op](handle, A, A, B, N)
    finally:
        handle.set_policy(None)
    assert np.array_equal(A.export(), want)
    A.destroy(), B.destroy(), pol.destroy()


@pytest.mark.parametrize("shape", [(64, 32, 64, 32), (2048, 1024, 2048, 1024), (512, 512, 512, 512),
                                   (256, 96, 256, 96), (384, 192, 384, 192), (160, 160, 160, 160),
                                   (4096, 2080, 4096, 2080), (8192, 4096, 8192, 4096), (128, 128, 64, 96)])
def test_divmod(handle, shape):
    bq, br, ba, bb = shape
    count = 1000
    a = _rows(9, count, ba)
    b = _rows(10, count, bb)
    b[:count // 2, -1] |= np.uint32(0x80000000)      # full-length divisors
    b[count // 2: count // 2 + 50, (bb // 64):] = 0  # divisors with leading zero limbs
    b[5] = 0                                         # division by zero
    q_want, r_want = oracle.divmod_(a, b, bq // 32, br // 32, count)
    A, B = handle.integers(ba, count, a), handle.integers(bb, count, b)
    Q, R = handle.integers(bq, count), handle.integers(br, count)
    xmp.divmod_(handle, Q, R, A, B, count)
    assert np.array_equal(Q.export(), q_want), shape
    assert np.array_equal(R.export(), r_want), shape
    # stream (digit) path forced
    pol = handle.policy()
    pol.set_algorithm(xmp.ALG_DIGITMP)
    handle.set_policy(pol)
    try:
        xmp.divmod_(handle, Q, R, A, B, count)
    finally:
        handle.set_policy(None)
    assert np.array_equal(Q.export(), q_want), (shape, "digit")
    assert np.array_equal(R.export(), r_want), (shape, "digit")
    for x in (A, B, Q, R):
        x.destroy()
    pol.destroy()


def test_divmod_indexed_in_place(handle):
    ba, bb, count = 512, 256, N
    a, b = _rows(11, count, ba), _rows(12, M, bb)
    qi, ri, ai, bi = _perm(13, count), _perm(14, count), _perm(15, count), _perm(16, M)
    q_want, r_want = oracle.divmod_(a, b, ba // 32, bb // 32, count, q_index=qi, r_index=ri, a_index=ai,
                                    b_index=bi, q_init=a)
    A, B, R = handle.integers(ba, count, a), handle.integers(bb, M, b), handle.integers(bb, count)
    pol = handle.policy()
    for k, idx in enumerate([qi, ri, ai, bi]):
        pol.set_indices(k, idx)
    handle.set_policy(pol)
    try:
        xmp.divmod_(handle, A, R, A, B, count)  # quotient written over the dividend
    finally:
        handle.set_policy(None)
    assert np.array_equal(A.export(), q_want)
    assert np.array_equal(R.export(), r_want)
    A.destroy(), B.destroy(), R.destroy(), pol.destroy()


@pytest.mark.parametrize("bits_out,bits_a", [(256, 256), (288, 256), (128, 256), (1024, 1024), (160, 96)])
def test_not_shf(handle, bits_out, bits_a):
    a = _rows(17, N, bits_a)
    rng = np.random.default_rng(18)
    shifts = rng.integers(-400, 400, size=M).astype(np.int32)
    A, C = handle.integers(bits_a, N, a), handle.integers(bits_out, N)
    if bits_out >= bits_a:
        xmp.not_(handle, C, A, N)
        assert np.array_equal(C.export(), oracle.not_(a, bits_out // 32, N))
    else:  # not needs an output at least as wide as its input (src/logic.cu:500-501)
        with pytest.raises(xmp.XmpError) as e:
            xmp.not_(handle, C, A, N)
        assert e.value.code == xmp.ERR["xmpErrorInvalidPrecision"]
    xmp.shf(handle, C, A, shifts, N)  # shf has no precision rule
    assert np.array_equal(C.export(), oracle.shf(a, shifts, bits_out // 32, N))
    if bits_out == bits_a:  # in place
        xmp.shf(handle, A, A, shifts, N)
        assert np.array_equal(A.export(), oracle.shf(a, shifts, bits_out // 32, N))
    A.destroy(), C.destroy()


@pytest.mark.parametrize("ba,bb", [(256, 256), (256, 128), (128, 256), (2048, 2048)])
def test_cmp_popc(handle, ba, bb):
    a, b = _rows(19, N, ba), _rows(20, M, bb)
    b[:10] = 0
    a[:50, :bb // 32] = b[:50, :ba // 32] if ba <= bb else np.pad(b[:50], ((0, 0), (0, 0)))[:, :min(ba, bb) // 32]
    A, B = handle.integers(ba, N, a), handle.integers(bb, M, b)
    assert np.array_equal(xmp.cmp(handle, A, B, N), oracle.cmp(a, b, N))
    assert np.array_equal(xmp.popc(handle, A, N), oracle.popc(a, N))
    ai = _perm(21, N)
    pol = handle.policy()
    pol.set_indices(0, ai)
    handle.set_policy(pol)
    try:
        assert np.array_equal(xmp.popc(handle, A, N), oracle.popc(a, N, a_index=ai))
        assert np.array_equal(xmp.cmp(handle, A, B, N), oracle.cmp(a, b, N, a_index=ai))
    finally:
        handle.set_policy(None)
    A.destroy(), B.destroy(), pol.destroy()


@pytest.mark.parametrize("size", [1, 2, 4, 8])
@pytest.mark.parametrize("order", [-1, 1])
@pytest.mark.parametrize("endian", [-1, 1])
def test_import_export_formats(handle, size, order, endian):
    bits, count = 256, 300
    words = bits // (8 * size)
    dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[size]
    raw = np.frombuffer(oracle.random_limbs(22, count, bits // 32).tobytes(), dtype=dt).reshape(count, words).copy()
    X = handle.integers(bits, count)
    X.import_(raw, words=words, order=order, size=size, endian=endian)
    # decode the wire format on the CPU
    vals = []
    for row in raw:
        ws = list(row) if order == -1 else list(row)[::-1]
        v = 0
        for k, w in enumerate(ws):
            w = int(w)
            if endian == 1:
                w = int.from_bytes(w.to_bytes(size, "little"), "big")
            v |= w << (8 * size * k)
        vals.append(v)
    assert ints_from_rows(X.export()) == vals
    back = X.export(order=order, size=size, endian=endian)
    assert np.array_equal(back, raw)
    X.destroy()


def test_import_export_nails_and_indices(handle):
    bits, count = 128, 64
    raw = oracle.random_limbs(23, count, 4)
    X = handle.integers(bits, count)
    X.import_(raw, nails=4)
    assert np.array_equal(X.export(), raw & np.uint32(0x0fffffff))
    gi = _perm(24, count)
    pol = handle.policy()
    pol.set_indices(0, gi)
    handle.set_policy(pol)
    try:
        X.import_(raw)                        # gathers wire row gi[i] into element i
        got_scatter = X.export()              # scatters element i to wire row gi[i]
    finally:
        handle.set_policy(None)
    assert np.array_equal(X.export(), raw[gi])
    assert np.array_equal(got_scatter, raw)
    X.destroy(), pol.destroy()


def test_set(handle):
    a = _rows(25, N, 512)
    A, B = handle.integers(512, N, a), handle.integers(512, N)
    lib = xmp.lib()
    xmp.check(lib.xmpIntegersSet(handle.h, B.x, A.x, N))
    assert np.array_equal(B.export(), a)
    oi, ii = _perm(26, M), _perm(27, M)
    pol = handle.policy()
    pol.set_indices(0, oi)
    pol.set_indices(1, ii)
    handle.set_policy(pol)
    try:
        C = handle.integers(512, N, np.zeros((N, 16), dtype=np.uint32))
        xmp.check(lib.xmpIntegersSet(handle.h, C.x, A.x, M))
    finally:
        handle.set_policy(None)
    want = np.zeros((N, 16), dtype=np.uint32)
    for i in range(M):
        want[oi[i]] = a[ii[i] % N]
    assert np.array_equal(C.export(), want)
    for x in (A, B, C):
        x.destroy()
    pol.destroy()


def test_error_codes(handle):
    lib = xmp.lib()
    A, B = handle.integers(256, 10), handle.integers(512, 10)
    small = handle.integers(128, 10)
    with pytest.raises(xmp.XmpError) as e:
        xmp.add(handle, small, A, B, 10)
    assert e.value.code == xmp.ERR["xmpErrorInvalidPrecision"]
    with pytest.raises(xmp.XmpError) as e:
        xmp.add(handle, A, A, A, 11)
    assert e.value.code == xmp.ERR["xmpErrorInvalidCount"]
    xmp.add(handle, B, A, A, 0)  # count 0 is a no-op
    with pytest.raises(xmp.XmpError) as e:
        handle.integers(100, 10)
    assert e.value.code == xmp.ERR["xmpErrorUnsupported"]
    with pytest.raises(xmp.XmpError) as e:
        handle.integers(256, 0)
    assert e.value.code == xmp.ERR["xmpErrorInvalidCount"]
    with pytest.raises(xmp.XmpError) as e:
        xmp.powm(handle, A, A, A, B, 10)
    assert e.value.code == xmp.ERR["xmpErrorInvalidPrecision"]
    with pytest.raises(xmp.XmpError) as e:
        A.import_(np.zeros((10, 4), dtype=np.uint32))  # 128 bits into a 256-bit array
    assert e.value.code == xmp.ERR["xmpErrorInvalidPrecision"]
    pol = handle.policy()
    with pytest.raises(xmp.XmpError) as e:
        pol.set_indices(4, [0])
    assert e.value.code == xmp.ERR["xmpErrorInvalidParameter"]
    pol.set_scratch_limit(1 << 20)
    assert pol.get(xmp.PARAM_SCRATCH_LIMIT) == 1 << 20
    pol.set_algorithm(xmp.ALG_REGMP)
    assert pol.get(xmp.PARAM_ALGORITHM) == xmp.ALG_REGMP
    handle.set_policy(pol)
    try:
        big = handle.integers(4096, 10)
        with pytest.raises(xmp.XmpError) as e:
            xmp.powm(handle, big, big, big, big, 10)  # per-thread registers stop at 1024 bits
        assert e.value.code == xmp.ERR["xmpErrorUnsupported"]
        big.destroy()
    finally:
        handle.set_policy(None)
    # scratch limit too small for any window table (import first: it stages host data through scratch);
    # 1,024 instances go to the lane kernels, whose tables live in scratch
    x = handle.integers(1024, 1024, oracle.full_length_odd(1, 1024, 32))
    ym = oracle.full_length_odd(2, 16, 32)
    y, yo = handle.integers(1024, 16, ym), handle.integers(1024, 16)
    tiny = handle.policy()
    tiny.set_scratch_limit(64)
    handle.set_policy(tiny)
    try:
        with pytest.raises(xmp.XmpError) as e:
            xmp.powm(handle, x, x, x, x, 1024)
        assert e.value.code == xmp.ERR["xmpErrorIncreaseScratchLimit"]
        # a small batch runs one instance per CTA with its table in shared memory: no scratch needed
        xmp.powm(handle, yo, y, y, y, 16)
    finally:
        handle.set_policy(None)
    want, _ = oracle.powm(ym, ym, ym, 16)
    assert np.array_equal(yo.export(), want)
    for v in (x, y, yo):
        v.destroy()
    dev = np.zeros(1, dtype=np.int32)
    import ctypes
    d = ctypes.c_int32(-1)
    xmp.check(lib.xmpHandleGetDevice(handle.h, ctypes.byref(d)))
    assert d.value >= 0
    for x in (A, B, small):
        x.destroy()
    pol.destroy(), tiny.destroy()


def test_full_size_add_sub_roundtrip(handle):
    """2^22 pairs of 256-bit integers: (a + b) - b == a and a ^ b ^ b == a at the elementwise suite's size."""
    n = 1 << 22
    a, b = oracle.random_limbs(30, n, 8), oracle.random_limbs(31, n, 8)
    A, B, S = handle.integers(256, n, a), handle.integers(256, n, b), handle.integers(256, n)
    xmp.add(handle, S, A, B, n)
    xmp.sub(handle, S, S, B, n)
    assert np.array_equal(S.export(), a)
    xmp.xor(handle, S, A, B, n)
    xmp.xor(handle, S, S, B, n)
    assert np.array_equal(S.export(), a)
    sample = np.arange(0, n, 4099)
    xmp.add(handle, S, A, B, n)
    got = S.export()[sample]
    assert np.array_equal(got, oracle.binary("add", a[sample], b[sample], 8, len(sample)))
    for x in (A, B, S):
        x.destroy()
