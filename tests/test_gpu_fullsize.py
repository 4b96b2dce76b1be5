"""Full-size parity for the measured workloads other than the headline.

* config 2 contraction ops at their measured sizes: 2^18 x 512 x 512 -> 1024-bit
  mul and 2^18 x 2048 / 1024-bit divmod (divisor top bit set), every instance
  against GMP (mpz_mul, mpz_tdiv_qr under OpenMP);
* config 3: the uneven-size batch at full size -- 65,536 instances (40/30/20/10%
  of 1024/2048/3072/4096-bit moduli, full-length exponents, bases below the
  moduli) plus 16,384 CRT-RSA-2048 private operations under 256 keys from
  mpz_nextprime -- through one batch plan; per bin a spread sample against GMP
  mpz_powm, every CRT result against its message, and the plan's plain items
  against plain xmpIntegersPowm on every instance.
The headline (65,536 x 2048) and the 4,096 x 1024-bit workload are checked in
test_gpu_powm.py and test_gpu_reference.py.
"""
import numpy as np
import pytest

import oracle
import xmp_b200 as xmp
from tests.test_gpu_batch import _keys

pytestmark = pytest.mark.gpu


def test_mul_512x512_2p18_all_instances(handle):
    M = 1 << 18
    a = oracle.random_limbs(41, M, 16)
    b = oracle.random_limbs(42, M, 16)
    A, B, C = handle.integers(512, M, a), handle.integers(512, M, b), handle.integers(1024, M)
    try:
        xmp.mul(handle, C, A, B, M)
        got = C.export()
    finally:
        for v in (A, B, C):
            v.destroy()
    assert np.array_equal(got, oracle.binary("mul", a, b, 32, M))


def test_divmod_2048_by_1024_2p18_all_instances(handle):
    M = 1 << 18
    a = oracle.random_limbs(51, M, 64)
    b = oracle.random_limbs(52, M, 32)
    b[:, -1] |= np.uint32(0x80000000)
    A, B, Q, R = handle.integers(2048, M, a), handle.integers(1024, M, b), handle.integers(2048, M), \
        handle.integers(1024, M)
    try:
        xmp.divmod_(handle, Q, R, A, B, M)
        q, r = Q.export(), R.export()
    finally:
        for v in (A, B, Q, R):
            v.destroy()
    wq, wr = oracle.divmod_(a, b, 64, 32, M)
    assert np.array_equal(q, wq)
    assert np.array_equal(r, wr)


def test_mixed_batch_full_size(handle):
    total, ncrt, nkeys = 65536, 16384, 256
    mix = [(1024, 0.4), (2048, 0.3), (3072, 0.2), (4096, 0.1)]
    sizes = [(b, int(total * f)) for b, f in mix]
    sizes[0] = (1024, total - sum(c for _, c in sizes[1:]))
    arrays, groups = [], []
    for k, (bits, cnt) in enumerate(sizes):
        n = bits // 32
        m = oracle.full_length_odd(900 + k, cnt, n)
        x = oracle.below(910 + k, m)
        e = oracle.random_limbs(920 + k, cnt, n)
        e[:, -1] |= np.uint32(0x80000000)
        X, E, Mo = (handle.integers(bits, cnt, v) for v in (x, e, m))
        O1, O2 = handle.integers(bits, cnt), handle.integers(bits, cnt)
        arrays += [X, E, Mo, O1, O2]
        groups.append(dict(bits=bits, count=cnt, x=x, e=e, m=m, X=X, E=E, M=Mo, O1=O1, O2=O2))
    keys = _keys(nkeys, 1024, 777)
    rng = np.random.default_rng(778)
    msgs, cts = [], []
    for i in range(ncrt):
        kk = keys[i % nkeys]
        nn = oracle.to_int(kk["n"])
        mm = int.from_bytes(rng.bytes(256), "little") % nn
        msgs.append(mm)
        cts.append(pow(mm, 65537, nn))
    C = handle.integers(2048, ncrt, np.stack([oracle.from_int(c, 64) for c in cts]))
    ka = {f: handle.integers(1024, nkeys, np.stack([kk[f] for kk in keys])) for f in ("p", "q", "dp", "dq", "qinv")}
    out = handle.integers(2048, ncrt)
    arrays += [C, out] + list(ka.values())
    try:
        plan = xmp.BatchPlan(handle, [(g["O2"], g["X"], g["E"], g["M"], g["count"]) for g in groups],
                             [(out, C, ka["p"], ka["q"], ka["dp"], ka["dq"], ka["qinv"], ncrt)], use_graph=True)
        plan.execute()
        for g in groups:
            xmp.powm(handle, g["O1"], g["X"], g["E"], g["M"], g["count"])
            got = g["O2"].export()
            assert np.array_equal(got, g["O1"].export()), g["bits"]
            idx = np.linspace(0, g["count"] - 1, 128).astype(np.int64)
            want, _ = oracle.powm(g["x"][idx], g["e"][idx], g["m"][idx], len(idx))
            assert np.array_equal(got[idx], want), g["bits"]
        res = out.export()
        assert [oracle.to_int(r) for r in res] == msgs
        plan.destroy()
    finally:
        for a in arrays:
            a.destroy()
