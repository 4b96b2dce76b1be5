"""Pins the CPU oracle (tests only, no GPU).

The oracle is checked against every golden vector in tests/golden/golden.json
(Python-integer expected values, including the reference's own 512-bit
Montgomery regression case and the toy CRT-RSA key of the samples), against
Python integer arithmetic on seeded random inputs with index and broadcast
rules, and its plain-C Montgomery restatement of the reference algorithm is
checked against GMP.
"""
import random

import numpy as np
import pytest

import oracle
from tests.helpers import cases, hexs, ints_from_rows, rows_from_ints


def _nl(bits):
    return bits // 32


@pytest.mark.parametrize("op", ["add", "sub", "and", "ior", "xor", "mul"])
def test_binary_golden(golden, op):
    for c in cases(golden, op):
        bo, ba, bb = c["precisions"]
        a, b = hexs(c["inputs"][0]), hexs(c["inputs"][1])
        want = hexs(c["outputs"][0])
        got = oracle.binary(op, rows_from_ints(a, _nl(ba)), rows_from_ints(b, _nl(bb)), _nl(bo), len(a))
        assert ints_from_rows(got) == want, (op, c["precisions"])


def test_not_golden(golden):
    for c in cases(golden, "not"):
        bo, ba = c["precisions"]
        a = hexs(c["inputs"][0])
        got = oracle.not_(rows_from_ints(a, _nl(ba)), _nl(bo), len(a))
        assert ints_from_rows(got) == hexs(c["outputs"][0])


def test_divmod_golden(golden):
    for c in cases(golden, "divmod"):
        bq, br, ba, bb = c["precisions"]
        a, b = hexs(c["inputs"][0]), hexs(c["inputs"][1])
        q, r = oracle.divmod_(rows_from_ints(a, _nl(ba)), rows_from_ints(b, _nl(bb)), _nl(bq), _nl(br), len(a))
        assert ints_from_rows(q) == hexs(c["outputs"][0])
        assert ints_from_rows(r) == hexs(c["outputs"][1])
        qd = oracle.binary("div", rows_from_ints(a, _nl(ba)), rows_from_ints(b, _nl(bb)), _nl(bq), len(a))
        rm = oracle.binary("mod", rows_from_ints(a, _nl(ba)), rows_from_ints(b, _nl(bb)), _nl(br), len(a))
        assert ints_from_rows(qd) == hexs(c["outputs"][0])
        assert ints_from_rows(rm) == hexs(c["outputs"][1])


def test_shf_golden(golden):
    for c in cases(golden, "shf"):
        bo, ba = c["precisions"]
        a, s = hexs(c["inputs"][0]), c["inputs"][1]
        got = oracle.shf(rows_from_ints(a, _nl(ba)), s, _nl(bo), len(a))
        assert ints_from_rows(got) == hexs(c["outputs"][0])


def test_cmp_popc_golden(golden):
    for c in cases(golden, "cmp"):
        ba, bb = c["precisions"]
        a, b = hexs(c["inputs"][0]), hexs(c["inputs"][1])
        got = oracle.cmp(rows_from_ints(a, _nl(ba)), rows_from_ints(b, _nl(bb)), len(a))
        assert list(got) == c["outputs"][0]
    for c in cases(golden, "popc"):
        (ba,) = c["precisions"]
        a = hexs(c["inputs"][0])
        assert list(oracle.popc(rows_from_ints(a, _nl(ba)), len(a))) == c["outputs"][0]


def test_powm_golden(golden):
    for c in cases(golden, "powm"):
        bo, bb, be, bm = c["precisions"]
        x, e, m = (hexs(v) for v in c["inputs"])
        want = hexs(c["outputs"][0])
        X, E, M = rows_from_ints(x, _nl(bb)), rows_from_ints(e, _nl(be)), rows_from_ints(m, _nl(bm))
        got, _ = oracle.powm(X, E, M, len(x))
        assert ints_from_rows(got) == want, c["precisions"]
        sec, _ = oracle.powm(X, E, M, len(x), sec=True)
        assert ints_from_rows(sec) == want
        mont = oracle.powm_mont(X, E, M, len(x))
        assert ints_from_rows(mont) == want, ("mont", c["precisions"])


def test_reference_regression_case(golden):
    c = [c for c in golden["cases"] if c.get("source", "").startswith("src/include/regmp/reduce_xmad.h")][0]
    x, e, m = (hexs(v)[0] for v in c["inputs"])
    assert hexs(c["outputs"][0])[0] == pow(x, e, m)


def test_crt_toy_key(golden):
    k = golden["crt_toy"]
    assert k["p"] * k["q"] == k["n"]
    ct = k["ciphertexts"]
    n_rows = rows_from_ints(ct, 1)
    p = rows_from_ints([k["p"]], 1)
    q = rows_from_ints([k["q"]], 1)
    # decrypt with the CRT sequence of the sample: mod, powm, mul, add, mod
    cm_p = oracle.binary("mod", n_rows, p, 1, len(ct))
    mp, _ = oracle.powm(cm_p, rows_from_ints([k["dp"]], 1), p, len(ct))
    cm_q = oracle.binary("mod", n_rows, q, 1, len(ct))
    mq, _ = oracle.powm(cm_q, rows_from_ints([k["dq"]], 1), q, len(ct))
    sp = oracle.binary("mul", mp, rows_from_ints([k["cp"]], 1), 2, len(ct))
    sq = oracle.binary("mul", mq, rows_from_ints([k["cq"]], 1), 2, len(ct))
    s = oracle.binary("add", sp, sq, 2, len(ct))
    r = oracle.binary("mod", s, rows_from_ints([k["n"]], 2), 2, len(ct))
    assert ints_from_rows(r) == k["messages"]


def test_index_and_broadcast_rules():
    """Output element out_index[i]; inputs index[i % n] % array_count (docs 15-16)."""
    rnd = random.Random(5)
    count, na, nb = 50, 13, 7
    a = [rnd.getrandbits(128) for _ in range(na)]
    b = [rnd.getrandbits(128) for _ in range(nb)]
    oi = list(range(count))
    rnd.shuffle(oi)
    ai = [rnd.randrange(1000) for _ in range(9)]
    bi = [rnd.randrange(1000) for _ in range(count)]
    got = oracle.binary("add", rows_from_ints(a, 4), rows_from_ints(b, 4), 5, count, out_index=oi, a_index=ai,
                        b_index=bi)
    want = [0] * count
    for i in range(count):
        want[oi[i]] = a[ai[i % len(ai)] % na] + b[bi[i % len(bi)] % nb]
    assert ints_from_rows(got) == want


@pytest.mark.parametrize("bits", [32, 96, 256, 1024])
def test_montgomery_restatement_vs_gmp(bits):
    n = bits // 32
    count = 24
    m = oracle.full_length_odd(11 + bits, count, n)
    m[0] = 0
    m[0, 0] = 1  # m = 1
    m[1, -1] = 0
    m[1, 0] |= 1  # top limb clear
    x = oracle.random_limbs(12 + bits, count, n)
    e = oracle.random_limbs(13 + bits, count, n)
    e[2] = 0
    g, _ = oracle.powm(x, e, m, count)
    mo = oracle.powm_mont(x, e, m, count)
    assert np.array_equal(g, mo)
    for i in range(4):
        assert oracle.to_int(g[i]) == pow(oracle.to_int(x[i]), oracle.to_int(e[i]), oracle.to_int(m[i]))


def test_generators_deterministic():
    a = oracle.full_length_odd(1, 8, 32)
    b = oracle.full_length_odd(1, 8, 32)
    assert np.array_equal(a, b)
    assert all(r[0] & 1 and r[-1] >> 31 for r in a)
    x = oracle.below(2, a)
    assert all(oracle.to_int(xi) < oracle.to_int(mi) for xi, mi in zip(x, a))


def test_crt_key_generation():
    p0 = oracle.random_limbs(3, 1, 4)[0]
    q0 = oracle.random_limbs(4, 1, 4)[0]
    p0[-1] |= 0x80000000
    q0[-1] |= 0x80000000
    k = oracle.crt_key(p0, q0)
    assert k is not None
    p, q = oracle.to_int(k["p"]), oracle.to_int(k["q"])
    assert oracle.to_int(k["n"]) == p * q
    assert (oracle.to_int(k["qinv"]) * q) % p == 1
    e = 65537
    msg = 123456789
    c = pow(msg, e, p * q)
    mp = pow(c % p, oracle.to_int(k["dp"]), p)
    mq = pow(c % q, oracle.to_int(k["dq"]), q)
    h = (oracle.to_int(k["qinv"]) * (mp - mq)) % p
    assert mq + q * h == msg
