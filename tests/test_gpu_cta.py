"""The CTA distribution (one exponentiation per CTA, xmp_b200/csrc/cta.cuh):
forced through xmpIntegersPowmWithConfigAsync (distribution 2) at every
supported operand size and at precisions padded up to one, against GMP, with
the edge moduli, bases and exponents of the lane-kernel tests; index arrays and
in-place output through the public call; the default choice for small and
large batches; and the server, whose small waves run the constant-schedule
form of the same kernel."""
import numpy as np
import pytest

import oracle
import xmp_b200 as xmp

pytestmark = pytest.mark.gpu


def _case(seed, count, bits, ebits=None):
    n = bits // 32
    m = oracle.full_length_odd(seed, count, n)
    x = oracle.random_limbs(seed + 1, count, n)  # bases anywhere below 2^bits (also >= m)
    e = oracle.random_limbs(seed + 2, count, (ebits or bits) // 32)
    return x, e, m


def _edges(x, e, m):
    m[0] = 0
    m[0, 0] = 1                  # m = 1
    m[1, :] = 0xffffffff         # all ones
    m[2, -1] = 0                 # top limb clear
    m[2, 0] |= 1
    m[3, :] = 0
    m[3, 0] = 3                  # m = 3
    e[4] = 0                     # x^0
    e[5] = 0
    e[5, 0] = 1                  # x^1
    x[6] = 0                     # 0^e
    x[7] = m[7]                  # x == m
    x[8] = 0xffffffff            # x = 2^bits - 1 > m
    e[9] = 0
    e[9, -1] = 0x80000000        # a single top bit
    return x, e, m


def _run_cta(h, x, e, m, count, window=0):
    bits = m.shape[1] * 32
    X, E, M, O = h.integers(bits, count, x), h.integers(e.shape[1] * 32, count, e), h.integers(bits, count, m), \
        h.integers(bits, count)
    try:
        cfg = xmp.PowmConfig()
        cfg.distribution = 2
        cfg.window = window or xmp.powm_get_config(h, bits, e.shape[1] * 32, 1).window
        xmp.powm_with_config(h, O, X, E, M, count, cfg)
        return O.export()
    finally:
        for v in (X, E, M, O):
            v.destroy()


@pytest.mark.parametrize("bits", [32, 160, 544, 1024, 1056, 1536, 2048, 2080, 3072, 3104, 4096])
def test_cta_sizes_and_edges(handle, bits):
    count = 40
    x, e, m = _edges(*_case(900 + bits, count, bits))
    want, _ = oracle.powm(x, e, m, count)
    got = _run_cta(handle, x, e, m, count)
    bad = np.nonzero(~np.all(got == want, axis=1))[0]
    assert len(bad) == 0, "mismatch at %s (bits=%d)" % (bad[:8], bits)


@pytest.mark.parametrize("window", [1, 3, 7])
@pytest.mark.parametrize("ebits", [32, 2048, 4096])
def test_cta_windows_and_exponent_precisions(handle, window, ebits):
    count = 12
    x, e, m = _case(950 + window + ebits, count, 2048, ebits)
    want, _ = oracle.powm(x, e, m, count)
    assert np.array_equal(_run_cta(handle, x, e, m, count, window), want)


def test_cta_default_choice(handle):
    """Small batches go one instance per CTA by default; large ones to the lane kernels."""
    small = xmp.powm_get_config(handle, 2048, 2048, 1)
    assert small.distribution == 2 and small.limbs == 64
    assert xmp.powm_get_config(handle, 1536, 1536, 16).distribution == 2
    assert xmp.powm_get_config(handle, 2048, 2048, 65536).distribution == 0
    assert xmp.powm_get_config(handle, 8192, 8192, 1).distribution != 2  # beyond 4096 bits
    assert xmp.powm_get_config(handle, 512, 512, 1).distribution != 2  # small moduli: the lane kernels
    assert xmp.powm_get_config(handle, 544, 544, 1).distribution == 2


def test_cta_default_batch_limits(handle):
    """The batch sizes up to which one instance per CTA is the default (instances per SM, by the
    CTA operand size and the modulus precision) and the first size past each limit."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for bits, per_sm in ((768, 4), (1024, 6), (1536, 2), (2048, 3), (3072, 1), (4096, 1)):
        assert xmp.powm_get_config(handle, bits, bits, per_sm * sms).distribution == 2, bits
        assert xmp.powm_get_config(handle, bits, bits, per_sm * sms + 1).distribution != 2, bits


def test_cta_through_the_default_call_with_indices_and_in_place(handle):
    bits, count = 2048, 24
    x, e, m = _case(990, count, bits)
    pol = xmp.Policy(handle)
    perm = np.random.default_rng(991).permutation(count).astype(np.uint32)
    X, E, M = handle.integers(bits, count, x), handle.integers(bits, count, e), handle.integers(bits, count, m)
    try:
        pol.set_indices(1, perm)  # gathered bases
        handle.set_policy(pol)
        O = handle.integers(bits, count)
        xmp.powm(handle, O, X, E, M, count)
        want, _ = oracle.powm(x[perm], e, m, count)
        assert np.array_equal(O.export(), want)
        O.destroy()
        handle.set_policy(None)
        xmp.powm(handle, X, X, E, M, count)  # out == base
        want, _ = oracle.powm(x, e, m, count)
        assert np.array_equal(X.export(), want)
    finally:
        handle.set_policy(None)
        pol.destroy()
        for v in (X, E, M):
            v.destroy()


def test_cta_full_wave_of_ctas(handle):
    """More CTAs than the GPU holds at once (two per SM and beyond), every result against GMP."""
    bits, count = 1024, 1200
    x, e, m = _case(995, count, bits)
    want, _ = oracle.powm(x, e, m, count)
    assert np.array_equal(_run_cta(handle, x, e, m, count), want)
