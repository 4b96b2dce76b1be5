"""CUDA modular exponentiation vs the GMP oracle (mpz_powm), bit-exact.

Covers every distribution (per-thread registers, warp-distributed, digit-serial)
over the reference's precision grid (unit_tests/test.cu:2815-2910: 32..8192 bits
and the odd sizes 160..544, 1056, 2080), broadcast counts, shuffled index
policies, in-place outputs, short/zero exponents and the edge moduli (m = 1,
top bits clear, all ones).
"""
import numpy as np
import pytest

import oracle
import xmp_b200 as xmp

pytestmark = pytest.mark.gpu


def _case(seed, count, bits, ebits=None, full=True):
    n = bits // 32
    m = oracle.full_length_odd(seed, count, n) if full else oracle.random_limbs(seed, count, n) | np.uint32(1)
    x = oracle.random_limbs(seed + 1, count, n)  # not reduced: bases may exceed m, as in the reference tests
    e = oracle.random_limbs(seed + 2, count, (ebits or bits) // 32)
    return x, e, m


def _run(handle, x, e, m, count, alg=xmp.ALG_DEFAULT, indices=None, out_count=None):
    bits = m.shape[1] * 32
    X, E, M = (handle.integers(v.shape[1] * 32, v.shape[0], v) for v in (x, e, m))
    O = handle.integers(bits, out_count or count)
    pol = handle.policy()
    pol.set_algorithm(alg)
    if indices:
        for k, idx in indices.items():
            pol.set_indices(k, idx)
    handle.set_policy(pol)
    try:
        xmp.powm(handle, O, X, E, M, count)
    finally:
        handle.set_policy(None)
        pol.destroy()
    got = O.export()
    for v in (X, E, M, O):
        v.destroy()
    return got


SIZES = [32, 64, 128, 160, 192, 224, 256, 288, 320, 352, 384, 512, 544, 1024, 1056, 2048, 2080, 3072, 4096]


@pytest.mark.parametrize("bits", SIZES)
@pytest.mark.parametrize("alg", [xmp.ALG_DEFAULT, xmp.ALG_REGMP, xmp.ALG_DISTRIBUTEDMP])
def test_powm_sizes(handle, bits, alg):
    if alg == xmp.ALG_REGMP and bits > 1024:
        pytest.skip("per-thread registers hold at most 1024 bits")
    count = 300 if bits <= 1024 else 96
    x, e, m = _case(100 + bits, count, bits, full=(bits % 64 == 0))
    m[0] = 0
    m[0, 0] = 1                  # m = 1
    m[1, :] = 0xffffffff         # all ones
    m[2, -1] = 0                 # top limb clear
    m[2, 0] |= 1
    e[3] = 0                     # x^0
    x[4] = 0                     # 0^e
    x[5] = m[5]                  # x == m
    want, _ = oracle.powm(x, e, m, count)
    got = _run(handle, x, e, m, count, alg)
    bad = np.nonzero(~np.all(got == want, axis=1))[0]
    assert len(bad) == 0, "mismatch at %s of %d (bits=%d alg=%d)" % (bad[:8], count, bits, alg)


@pytest.mark.parametrize("bits", [64, 256, 544, 1056, 2080])
def test_powm_digit_serial(handle, bits):
    count = 64
    x, e, m = _case(200 + bits, count, bits)
    e[0] = 0
    want, _ = oracle.powm(x, e, m, count)
    assert np.array_equal(_run(handle, x, e, m, count, xmp.ALG_DIGITMP), want)


@pytest.mark.parametrize("bits", [6144, 8192])
def test_powm_large(handle, bits):
    count = 32
    x, e, m = _case(300 + bits, count, bits)
    e = e[:, :2].copy()  # short exponents keep the CPU oracle fast; scan length = exponent precision
    want, _ = oracle.powm(x, e, m, count)
    assert np.array_equal(_run(handle, x, e, m, count), want)
    assert np.array_equal(_run(handle, x, e, m, count, xmp.ALG_DISTRIBUTEDMP), want)


@pytest.mark.parametrize("ebits", [32, 64, 256, 1024, 2048])
def test_powm_exponent_precisions(handle, ebits):
    """Exponent precision differs from the modulus precision (src/powm.cu:268-269)."""
    bits, count = 1024, 256
    x, e, m = _case(400 + ebits, count, bits, ebits=ebits)
    e[::3, -1] = 0   # some exponents shorter than their precision
    e[1] = 0
    e[2] = 0
    e[2, 0] = 17
    want, _ = oracle.powm(x, e, m, count)
    assert np.array_equal(_run(handle, x, e, m, count), want)


@pytest.mark.parametrize("counts", [(2000, 2000, 2000, 2000, 2000), (2000, 2000, 1, 1, 2000),
                                    (2000, 100, 100, 100, 2000), (2000, 1, 100, 2000, 2000),
                                    (2000, 2000, 2000, 2000, 100), (2000, 2000, 4000, 2000, 2000)])
@pytest.mark.parametrize("alg", [xmp.ALG_DEFAULT, xmp.ALG_DISTRIBUTEDMP, xmp.ALG_REGMP])
def test_powm_indices_broadcast(handle, counts, alg):
    """The reference's PowmParams grid (c, b, e, m counts, op count) with shuffled index arrays."""
    cN, bN, eN, mN, n = counts
    bits = 128
    rng = np.random.default_rng(sum(counts))
    x = oracle.random_limbs(1, bN, 4)
    e = oracle.random_limbs(2, eN, 4)
    m = oracle.random_limbs(3, mN, 4) | np.uint32(1)
    idx = {0: rng.permutation(cN).astype(np.uint32), 1: rng.permutation(bN).astype(np.uint32),
           2: rng.permutation(eN).astype(np.uint32), 3: rng.permutation(mN).astype(np.uint32)}
    want, _ = oracle.powm(x, e, m, n, out_count=cN, out_index=idx[0], base_index=idx[1], exp_index=idx[2],
                          mod_index=idx[3])
    got = _run(handle, x, e, m, n, alg, indices=idx, out_count=cN)
    written = idx[0][:n]
    assert np.array_equal(got[written], want[written])


def test_powm_in_place(handle):
    bits, count = 512, 1000
    x, e, m = _case(500, count, bits)
    want, _ = oracle.powm(x, e, m, count)
    X, E, M = (handle.integers(bits, count, v) for v in (x, e, m))
    xmp.powm(handle, X, X, E, M, count)
    assert np.array_equal(X.export(), want)
    # in place with indices (the reference's in-place test, unit_tests/test.cu:1231-1252)
    X.import_(x)
    oi = np.random.default_rng(1).permutation(count).astype(np.uint32)
    bi = np.random.default_rng(2).permutation(count).astype(np.uint32)
    want2, _ = oracle.powm(x, e, m, count, out_index=oi, base_index=bi, init=x)
    pol = handle.policy()
    pol.set_indices(0, oi)
    pol.set_indices(1, bi)
    handle.set_policy(pol)
    try:
        xmp.powm(handle, X, X, E, M, count)
    finally:
        handle.set_policy(None)
    assert np.array_equal(X.export(), want2)
    # exponent overwritten by the result
    E.import_(e)
    xmp.powm(handle, E, X, E, M, count)
    want3, _ = oracle.powm(want2, e, m, count)
    assert np.array_equal(E.export(), want3)
    for v in (X, E, M):
        v.destroy()
    pol.destroy()


def _special_exponents(count, nlimbs, seed):
    """Exponents that stress a sliding-window scan, interleaved so the instances of one warp
    follow different schedules: 0, 1, 2, powers of two (trailing zeros), all ones, alternating
    bits, long zero runs between ones, one-limb and full random values."""
    e = oracle.random_limbs(seed, count, nlimbs)
    top = nlimbs * 32 - 1
    for r in range(count):
        kind = r % 11
        v = None
        if kind == 0:
            v = 0
        elif kind == 1:
            v = 1
        elif kind == 2:
            v = 2
        elif kind == 3:
            v = 1 << (r * 7 % (top + 1))
        elif kind == 4:
            v = (1 << (top + 1)) - 1
        elif kind == 5:
            v = int("01" * ((top + 1) // 2), 2)
        elif kind == 6:
            v = int("10" * ((top + 1) // 2), 2)
        elif kind == 7:
            v = (1 << top) | (1 << (top // 2)) | 1
        elif kind == 8:
            v = int(e[r, 0])  # one limb
        elif kind == 9:
            v = (1 << top) | (0b1000001 << (r % (top - 8)))
        if v is not None:
            e[r] = [(v >> (32 * k)) & 0xFFFFFFFF for k in range(nlimbs)]
    return e


@pytest.mark.parametrize("lanes,limbs", [(2, 8), (4, 5), (8, 4), (16, 2), (1, 8), (8, 1)])
def test_powm_window_schedules(handle, lanes, limbs):
    """Every window size 1..7 of a register kernel, with exponents whose schedules differ within a
    warp.  2 x 8, 4 x 5, 8 x 4 and 16 x 2 run the sliding window (instances that finish early
    multiply by Mont(1) until the warp is done), 1 x 8 and 8 x 1 the fixed window."""
    bits = lanes * limbs * 32
    count = 200
    m = oracle.full_length_odd(700 + bits, count, bits // 32)
    x = oracle.below(701 + bits, m)
    e = _special_exponents(count, bits // 32, 702 + bits)
    want, _ = oracle.powm(x, e, m, count)
    X, E, M = (handle.integers(bits, count, v) for v in (x, e, m))
    O = handle.integers(bits, count)
    try:
        for w in range(1, 8):
            cfg = xmp.PowmConfig(0, lanes, limbs, w)
            xmp.powm_with_config(handle, O, X, E, M, count, cfg)
            got = O.export()
            bad = np.nonzero(~np.all(got == want, axis=1))[0]
            assert len(bad) == 0, "window %d: mismatch at %s" % (w, bad[:8])
    finally:
        for v in (X, E, M, O):
            v.destroy()


def test_powm_every_registered_config(handle):
    """Each (lanes, limbs per lane) kernel at its own capacity, through the default path with a forced config."""
    import ctypes
    # exercised indirectly: sizes chosen so the heuristic lands on different distributions
    for bits, count in [(96, 40000), (320, 3000), (1024, 64), (1024, 20000), (2048, 4096), (4096, 512)]:
        x, e, m = _case(600 + bits, count, bits)
        e = e[:, :1].copy()
        want, _ = oracle.powm(x, e, m, count)
        assert np.array_equal(_run(handle, x, e, m, count), want), bits


def test_powm_bench_workload_sample(handle):
    """2048-bit powm at the benchmark's batch (65,536 instances): a seeded sample is checked against GMP."""
    bits, count = 2048, 65536
    m = oracle.full_length_odd(7, count, 64)
    x = oracle.below(8, m)
    e = oracle.random_limbs(9, count, 64)
    e[:, -1] |= np.uint32(0x80000000)
    got = _run(handle, x, e, m, count)
    sample = np.arange(0, count, 997)
    want, _ = oracle.powm(x[sample], e[sample], m[sample], len(sample))
    assert np.array_equal(got[sample], want)


@pytest.mark.parametrize("lanes,limbs", [(4, 4), (4, 8), (4, 12), (4, 16), (1, 1), (1, 2), (1, 5), (1, 8),
                                         (1, 12), (1, 16)])
def test_powm_squaring_shapes(handle, lanes, limbs):
    """The shapes whose squarings use the specialised product (four-lane blocks fed into the reduction,
    per-thread separated scanning), at several windows, with full-length moduli, moduli whose top limbs
    are zero, bases 0, 1 and m - 1 and all-ones exponents."""
    bits = lanes * limbs * 32
    n = bits // 32
    count = 320
    m = oracle.full_length_odd(900 + bits, count, n)
    m[1::4, n // 2:] = 0  # a quarter of the moduli with their top half zero
    m[1::4, max(0, n // 2 - 1)] |= np.uint32(1 << 31) if n > 1 else np.uint32(0)
    m[:, 0] |= np.uint32(1)
    x = oracle.below(901 + bits, m)
    x[2::16] = 0
    x[3::16] = 0
    x[3::16, 0] = 1
    x[5::16] = m[5::16]
    x[5::16, 0] -= np.uint32(1)
    e = oracle.random_limbs(902 + bits, count, n)
    e[7::16] = 0xFFFFFFFF
    want, _ = oracle.powm(x, e, m, count)
    X, E, M = (handle.integers(bits, count, v) for v in (x, e, m))
    O = handle.integers(bits, count)
    try:
        for w in (1, 3, 6):
            xmp.powm_with_config(handle, O, X, E, M, count, xmp.PowmConfig(0, lanes, limbs, w))
            got = O.export()
            bad = np.nonzero(~np.all(got == want, axis=1))[0]
            assert len(bad) == 0, "window %d: mismatch at %s" % (w, bad[:8])
    finally:
        for v in (X, E, M, O):
            v.destroy()


@pytest.mark.parametrize("bits,alg", [(12288, xmp.ALG_DEFAULT), (16384, xmp.ALG_DEFAULT),
                                      (16384, xmp.ALG_DIGITMP), (20480, xmp.ALG_DEFAULT),
                                      (32768, xmp.ALG_DEFAULT)])
def test_powm_beyond_8192_bits(handle, bits, alg):
    """Above the reference's largest tuned precision (8192 bits, src/powm.cu:61): the register kernels
    up to 16,384 bits (32 lanes x 12 / 16 limbs) and the digit-serial kernel beyond, which the
    reference also uses past its tables (src/powm.cu:197-208).  Short exponents keep GMP fast."""
    count = 8
    x, e, m = _case(400 + bits // 32, count, bits)
    e = e[:, :2].copy()
    e[0] = 0
    e[1, 1] = 0xFFFFFFFF
    want, _ = oracle.powm(x, e, m, count)
    assert np.array_equal(_run(handle, x, e, m, count, alg), want)
