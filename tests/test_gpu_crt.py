"""The fused CRT-RSA operation (xmpIntegersPowmCRT): one kernel for c mod p, c
mod q, both half exponentiations and Garner's recombination, checked as an RSA
decryption (m = c^d mod pq recovers the message encrypted with e = 65537) and
against GMP mpz_powm of c^d mod n computed from the same key; keys from GMP
mpz_nextprime at several sizes, the reference sample's toy key (top bits of p
and q clear), exponent arrays of other precisions, broadcast keys, errors."""
import math

import numpy as np
import pytest

import oracle
import xmp_b200 as xmp
from tests.test_gpu_batch import _keys

pytestmark = pytest.mark.gpu


def _decrypt(h, keys, cts, half_bits, dexp_bits=None):
    hn = half_bits // 32
    count, nkeys = len(cts), len(keys)
    rows = {k: np.stack([kk[k] for kk in keys]) for k in ("p", "q", "dp", "dq", "qinv")}
    if dexp_bits:  # the same exponents held in arrays of another precision (one for both, or (dp, dq))
        for k, bits in zip(("dp", "dq"), dexp_bits if isinstance(dexp_bits, tuple) else (dexp_bits, dexp_bits)):
            r = np.zeros((nkeys, bits // 32), dtype=np.uint32)
            w = min(hn, bits // 32)
            r[:, :w] = rows[k][:, :w]
            rows[k] = r
    C = h.integers(2 * half_bits, count, np.stack([oracle.from_int(c, 2 * hn) for c in cts]))
    arr = {k: h.integers(32 * rows[k].shape[1], nkeys, rows[k]) for k in rows}
    O = h.integers(2 * half_bits, count)
    try:
        xmp.powm_crt(h, O, C, arr["p"], arr["q"], arr["dp"], arr["dq"], arr["qinv"], count)
        return [oracle.to_int(r) for r in O.export()]
    finally:
        for v in [C, O] + list(arr.values()):
            v.destroy()


@pytest.mark.parametrize("half_bits,count,nkeys", [(1024, 640, 16), (512, 1000, 7), (256, 333, 5), (1536, 96, 3),
                                                   (2048, 64, 2), (128, 200, 4)])
def test_crt_decrypts(handle, half_bits, count, nkeys):
    keys = _keys(nkeys, half_bits, 4000 + half_bits)
    rng = np.random.default_rng(half_bits)
    msgs, cts = [], []
    for i in range(count):
        n = oracle.to_int(keys[i % nkeys]["n"])
        m = int.from_bytes(rng.bytes(2 * half_bits // 8), "little") % n
        msgs.append(m)
        cts.append(pow(m, 65537, n))
    assert _decrypt(handle, keys, cts, half_bits) == msgs


def test_crt_matches_gmp_for_any_c_below_n(handle):
    """c uniform below n (not an encryption): out == c^d mod n with d from the key (GMP powm on n)."""
    half_bits, count, nkeys = 512, 256, 4
    keys = _keys(nkeys, half_bits, 4100)
    rng = np.random.default_rng(4101)
    cts, want = [], []
    for i in range(count):
        k = keys[i % nkeys]
        p, q = oracle.to_int(k["p"]), oracle.to_int(k["q"])
        n = p * q
        d = pow(65537, -1, (p - 1) * (q - 1) // math.gcd(p - 1, q - 1))
        c = int.from_bytes(rng.bytes(128), "little") % n
        cts.append(c)
        want.append(pow(c, d, n))
    assert _decrypt(handle, keys, cts, half_bits) == want


def test_crt_toy_key_and_exponent_precision(handle):
    """The reference sample's toy key (p = 4931, q = 3541 in 64-bit arrays: top bits clear), and the
    private exponents held in arrays wider than the primes."""
    p, q = 4931, 3541
    n = p * q
    d = pow(65537, -1, (p - 1) * (q - 1))
    key = {"p": oracle.from_int(p, 2), "q": oracle.from_int(q, 2), "dp": oracle.from_int(d % (p - 1), 2),
           "dq": oracle.from_int(d % (q - 1), 2), "qinv": oracle.from_int(pow(q, -1, p), 2), "n": oracle.from_int(n, 4)}
    msgs = [(i * 7919 + 13) % n for i in range(128)]
    cts = [pow(m, 65537, n) for m in msgs]
    assert _decrypt(handle, [key], cts, 64) == msgs
    assert _decrypt(handle, [key], cts, 64, dexp_bits=128) == msgs
    # dp and dq in arrays of different precisions: both halves of an operation scan the wider one
    assert _decrypt(handle, [key], cts, 64, dexp_bits=(32, 128)) == msgs
    assert _decrypt(handle, [key], cts, 64, dexp_bits=(96, 32)) == msgs


def test_crt_mixed_exponent_precisions_full_size_key(handle):
    """1024-bit halves with dq held in a 2048-bit array and dp in its own 1024-bit one."""
    keys = _keys(3, 1024, 4200)
    rng = np.random.default_rng(4201)
    msgs, cts = [], []
    for i in range(200):
        n = oracle.to_int(keys[i % 3]["n"])
        m = int.from_bytes(rng.bytes(256), "little") % n
        msgs.append(m)
        cts.append(pow(m, 65537, n))
    assert _decrypt(handle, keys, cts, 1024, dexp_bits=(1024, 2048)) == msgs


def test_crt_errors(handle):
    p = handle.integers(512, 4, oracle.full_length_odd(1, 4, 16))
    c, out_bad, out = handle.integers(1024, 4), handle.integers(768, 4), handle.integers(1024, 4)
    try:
        with pytest.raises(xmp.XmpError) as ei:
            xmp.powm_crt(handle, out_bad, c, p, p, p, p, p, 4)
        assert ei.value.name == "xmpErrorInvalidPrecision"
        with pytest.raises(xmp.XmpError) as ei:
            xmp.powm_crt(handle, out, c, p, p, p, p, p, 5)
        assert ei.value.name == "xmpErrorInvalidCount"
        xmp.powm_crt(handle, out, c, p, p, p, p, p, 0)  # count 0: nothing to do
    finally:
        for v in (p, c, out_bad, out):
            v.destroy()
