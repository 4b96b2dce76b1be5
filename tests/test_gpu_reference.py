"""Bit-exact parity with the reference XMP kernels themselves.

The reference library is built from its own sources for sm_100a by
oracle/build_ref.sh (oracle/_ref/libxmp_ref_imad.so, the -DIMAD variant) and
loaded next to libxmp.so; the same seeded inputs go through both C APIs and
the results must be identical, and identical to GMP.  Inputs stay inside the
launch shapes the reference runs with every lane active (oracle/ref_xmp.py):
instance counts in whole blocks of 128, full-length moduli and divisors.

The reference's documented defects (cmp of unequal precisions reads instance
0's high limbs, in-place indexed outputs) are not exercised here; they are
covered against the oracle's fixed rule in test_gpu_ops.py.
"""
import numpy as np
import pytest

import oracle
from oracle import ref_xmp
import xmp_b200 as xmp

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_xmp.available(), reason="reference library not built (oracle/build_ref.sh)")]


@pytest.fixture(scope="module")
def ref():
    r = ref_xmp.Ref("imad")
    yield r
    r.close()


@pytest.fixture(scope="module")
def ref_xmad():
    """The reference's default build (16-bit XMAD multiply emulation)."""
    if not ref_xmp.available("xmad"):
        pytest.skip("reference XMAD variant not built")
    r = ref_xmp.Ref("xmad")
    yield r
    r.close()


def _ours_powm(h, x, e, m):
    count, n = m.shape
    X, E, M, O = h.integers(32 * n, count, x), h.integers(32 * e.shape[1], count, e), h.integers(32 * n, count, m), \
        h.integers(32 * n, count)
    try:
        xmp.powm(h, O, X, E, M, count)
        return O.export()
    finally:
        for v in (X, E, M, O):
            v.destroy()


def _inputs(seed, bits, count, ebits=None, full=True):
    n = bits // 32
    if full:
        m = oracle.full_length_odd(seed, count, n)
    else:  # odd, any length above one limb
        m = oracle.random_limbs(seed, count, n)
        m[:, 0] |= np.uint32(1)
        m[:, -1] |= np.uint32(1)
    x = oracle.below(seed + 1, m)
    e = oracle.random_limbs(seed + 2, count, (ebits or bits) // 32)
    return x, e, m


def test_powm_config1_exact(handle, ref):
    """4,096 x 1024-bit, full-length exponents (the plain batched modexp workload): libxmp == reference == GMP."""
    from bench import make_inputs
    x, e, m = make_inputs(1024, 4096)
    ours = _ours_powm(handle, x, e, m)
    theirs = ref.powm(x, e, m)
    assert np.array_equal(ours, theirs)
    want, _ = oracle.powm(x, e, m, 4096)
    assert np.array_equal(ours, want)


def test_powm_xmad_variant(handle, ref_xmad):
    """The reference's default XMAD build gives the same results (1024 and 2048 bits)."""
    for bits, count in ((1024, 512), (2048, 256)):
        x, e, m = _inputs(700 + bits, bits, count)
        assert np.array_equal(_ours_powm(handle, x, e, m), ref_xmad.powm(x, e, m)), bits


@pytest.mark.parametrize("bits,count", [(2048, 1024), (1536, 512)])
def test_powm_distributed(handle, ref, bits, count):
    x, e, m = _inputs(100 + bits, bits, count)
    ours = _ours_powm(handle, x, e, m)
    assert np.array_equal(ours, ref.powm(x, e, m))
    want, _ = oracle.powm(x[:128], e[:128], m[:128], 128)
    assert np.array_equal(ours[:128], want)


@pytest.mark.parametrize("bits", [64, 128, 256, 384, 512])
def test_powm_per_thread(handle, ref, bits):
    """Up to 512 bits the reference runs its per-thread (RegMP) kernels; moduli need not be full length."""
    x, e, m = _inputs(200 + bits, bits, 512, full=False)
    ours = _ours_powm(handle, x, e, m)
    assert np.array_equal(ours, ref.powm(x, e, m))
    want, _ = oracle.powm(x, e, m, 512)
    assert np.array_equal(ours, want)


@pytest.mark.parametrize("bits,ebits", [(1024, 32), (1024, 64), (2048, 96), (512, 1024)])
def test_powm_exponent_precision(handle, ref, bits, ebits):
    """Exponent precision independent of the modulus': both scan the exponent over its precision."""
    x, e, m = _inputs(300 + bits + ebits, bits, 256, ebits=ebits)
    ours = _ours_powm(handle, x, e, m)
    assert np.array_equal(ours, ref.powm(x, e, m))
    want, _ = oracle.powm(x, e, m, 256)
    assert np.array_equal(ours, want)


def test_powm_edge_operands(handle, ref):
    """Bases 0, 1, m-1 and exponents 0, 1 (full-length 1024-bit moduli)."""
    count, n = 256, 32
    x, e, m = _inputs(400, 1024, count)
    x[0::8] = 0
    x[1::8] = 0
    x[1::8, 0] = 1
    mm1 = m.copy()
    mm1[:, 0] -= np.uint32(1)  # m is odd: m - 1 only touches the low limb
    x[2::8] = mm1[2::8]
    e[3::8] = 0
    e[4::8] = 0
    e[4::8, 0] = 1
    e[5::8] = 0xFFFFFFFF
    ours = _ours_powm(handle, x, e, m)
    assert np.array_equal(ours, ref.powm(x, e, m))
    want, _ = oracle.powm(x, e, m, count)
    assert np.array_equal(ours, want)


def _ours_binary(h, op, a, b, out_bits, count):
    A, B, C = h.integers(32 * a.shape[1], a.shape[0], a), h.integers(32 * b.shape[1], b.shape[0], b), \
        h.integers(out_bits, count)
    try:
        {"add": xmp.add, "sub": xmp.sub, "mul": xmp.mul, "ior": xmp.ior, "and": xmp.and_, "xor": xmp.xor}[op](
            h, C, A, B, count)
        return C.export()
    finally:
        for v in (A, B, C):
            v.destroy()


@pytest.mark.parametrize("op", ["add", "sub", "and", "ior", "xor"])
@pytest.mark.parametrize("bits_a,bits_b,bits_out", [(256, 256, 256), (256, 256, 288), (512, 256, 512),
                                                    (1024, 1024, 1024), (96, 96, 128)])
def test_elementwise(handle, ref, op, bits_a, bits_b, bits_out):
    """The config-2 element size (256 bits, wrapping and with a carry limb) and a few others."""
    count = 65536 if bits_a == 256 else 4096
    a = oracle.random_limbs(500, count, bits_a // 32)
    b = oracle.random_limbs(501, count, bits_b // 32)
    ours = _ours_binary(handle, op, a, b, bits_out, count)
    assert np.array_equal(ours, ref.binary(op, a, b, bits_out, count)), op
    assert np.array_equal(ours, oracle.binary(op, a, b, bits_out // 32, count)), op


def test_not_shf_cmp_popc(handle, ref):
    count, bits = 65536, 256
    a = oracle.random_limbs(510, count, 8)
    b = a.copy()
    b[::3] = oracle.random_limbs(511, count, 8)[::3]  # a third differ, the rest compare equal
    A, B = handle.integers(bits, count, a), handle.integers(bits, count, b)
    C = handle.integers(bits, count)
    try:
        xmp.not_(handle, C, A, count)
        assert np.array_equal(C.export(), ref.not_(a, bits, count))
        shifts = (np.random.default_rng(512).integers(-300, 300, size=count)).astype(np.int32)
        xmp.shf(handle, C, A, shifts, count)
        assert np.array_equal(C.export(), ref.shf(a, shifts, bits, count))
        assert np.array_equal(C.export(), oracle.shf(a, shifts, 8, count))
        got = xmp.cmp(handle, A, B, count)
        assert np.array_equal(got, ref.cmp(a, b, count))
        assert np.array_equal(got, oracle.cmp(a, b, count))
        got = xmp.popc(handle, A, count)
        assert np.array_equal(got, ref.popc(a, count))
    finally:
        for v in (A, B, C):
            v.destroy()


@pytest.mark.parametrize("bits_a,bits_b", [(512, 512), (256, 256), (1024, 512), (160, 96)])
def test_mul(handle, ref, bits_a, bits_b):
    """512 x 512 -> 1024 is the config-2 shape (the reference's digit-serial mul); the others its register mul."""
    count = 4096
    a = oracle.random_limbs(520 + bits_a, count, bits_a // 32)
    b = oracle.random_limbs(521 + bits_b, count, bits_b // 32)
    out_bits = bits_a + bits_b
    ours = _ours_binary(handle, "mul", a, b, out_bits, count)
    assert np.array_equal(ours, ref.binary("mul", a, b, out_bits, count))
    assert np.array_equal(ours, oracle.binary("mul", a, b, out_bits // 32, count))


@pytest.mark.parametrize("bits_a,bits_b", [(2048, 1024), (512, 256), (256, 128), (1024, 1024)])
def test_divmod(handle, ref, bits_a, bits_b):
    """2048 / 1024 with the divisor's top bit set is the config-2 shape (the reference's digit-serial division)."""
    count = 4096
    a = oracle.random_limbs(530 + bits_a, count, bits_a // 32)
    b = oracle.full_length_odd(531 + bits_b, count, bits_b // 32)
    A, B = handle.integers(bits_a, count, a), handle.integers(bits_b, count, b)
    Q, R = handle.integers(bits_a, count), handle.integers(bits_b, count)
    try:
        xmp.divmod_(handle, Q, R, A, B, count)
        q, r = Q.export(), R.export()
    finally:
        for v in (A, B, Q, R):
            v.destroy()
    rq, rr = ref.divmod_(a, b, count)
    assert np.array_equal(q, rq) and np.array_equal(r, rr)
    wq, wr = oracle.divmod_(a, b, bits_a // 32, bits_b // 32, count)
    assert np.array_equal(q, wq) and np.array_equal(r, wr)
