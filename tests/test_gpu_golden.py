"""Every golden vector through the CUDA path (libxmp.so via its C ABI)."""
import numpy as np
import pytest

import xmp_b200 as xmp
from tests.helpers import cases, hexs, ints_from_rows, rows_from_ints

pytestmark = pytest.mark.gpu


def _nl(bits):
    return bits // 32


def _arr(h, bits, vals):
    x = h.integers(bits, len(vals))
    x.import_(rows_from_ints(vals, _nl(bits)))
    return x


@pytest.mark.parametrize("op", ["add", "sub", "and", "ior", "xor", "mul"])
def test_binary(handle, golden, op):
    fn = {"add": xmp.add, "sub": xmp.sub, "and": xmp.and_, "ior": xmp.ior, "xor": xmp.xor, "mul": xmp.mul}[op]
    for c in cases(golden, op):
        bo, ba, bb = c["precisions"]
        a, b = hexs(c["inputs"][0]), hexs(c["inputs"][1])
        A, B, C = _arr(handle, ba, a), _arr(handle, bb, b), handle.integers(bo, len(a))
        fn(handle, C, A, B, len(a))
        assert ints_from_rows(C.export()) == hexs(c["outputs"][0]), (op, c["precisions"])
        for x in (A, B, C):
            x.destroy()


def test_not(handle, golden):
    for c in cases(golden, "not"):
        bo, ba = c["precisions"]
        a = hexs(c["inputs"][0])
        A, C = _arr(handle, ba, a), handle.integers(bo, len(a))
        xmp.not_(handle, C, A, len(a))
        assert ints_from_rows(C.export()) == hexs(c["outputs"][0])
        A.destroy(), C.destroy()


def test_divmod_div_mod(handle, golden):
    for c in cases(golden, "divmod"):
        bq, br, ba, bb = c["precisions"]
        a, b = hexs(c["inputs"][0]), hexs(c["inputs"][1])
        A, B = _arr(handle, ba, a), _arr(handle, bb, b)
        Q, R = handle.integers(bq, len(a)), handle.integers(br, len(a))
        xmp.divmod_(handle, Q, R, A, B, len(a))
        assert ints_from_rows(Q.export()) == hexs(c["outputs"][0]), c["precisions"]
        assert ints_from_rows(R.export()) == hexs(c["outputs"][1]), c["precisions"]
        Q2, R2 = handle.integers(bq, len(a)), handle.integers(br, len(a))
        xmp.div(handle, Q2, A, B, len(a))
        xmp.mod(handle, R2, A, B, len(a))
        assert ints_from_rows(Q2.export()) == hexs(c["outputs"][0])
        assert ints_from_rows(R2.export()) == hexs(c["outputs"][1])
        for x in (A, B, Q, R, Q2, R2):
            x.destroy()


def test_shf(handle, golden):
    for c in cases(golden, "shf"):
        bo, ba = c["precisions"]
        a, s = hexs(c["inputs"][0]), c["inputs"][1]
        A, C = _arr(handle, ba, a), handle.integers(bo, len(a))
        xmp.shf(handle, C, A, np.array(s, dtype=np.int32), len(a))
        assert ints_from_rows(C.export()) == hexs(c["outputs"][0]), c["precisions"]
        A.destroy(), C.destroy()


def test_cmp_popc(handle, golden):
    for c in cases(golden, "cmp"):
        ba, bb = c["precisions"]
        a, b = hexs(c["inputs"][0]), hexs(c["inputs"][1])
        A, B = _arr(handle, ba, a), _arr(handle, bb, b)
        assert list(xmp.cmp(handle, A, B, len(a))) == c["outputs"][0], c["precisions"]
        A.destroy(), B.destroy()
    for c in cases(golden, "popc"):
        (ba,) = c["precisions"]
        a = hexs(c["inputs"][0])
        A = _arr(handle, ba, a)
        assert list(xmp.popc(handle, A, len(a))) == c["outputs"][0]
        A.destroy()


@pytest.mark.parametrize("alg", [xmp.ALG_DEFAULT, xmp.ALG_REGMP, xmp.ALG_DISTRIBUTEDMP, xmp.ALG_DIGITMP])
def test_powm(handle, golden, alg):
    pol = handle.policy()
    pol.set_algorithm(alg)
    handle.set_policy(pol)
    try:
        for c in cases(golden, "powm"):
            bo, bb, be, bm = c["precisions"]
            if alg == xmp.ALG_REGMP and bm > 1024:
                continue
            x, e, m = (hexs(v) for v in c["inputs"])
            X, E, M, O = _arr(handle, bb, x), _arr(handle, be, e), _arr(handle, bm, m), handle.integers(bo, len(x))
            xmp.powm(handle, O, X, E, M, len(x))
            assert ints_from_rows(O.export()) == hexs(c["outputs"][0]), (alg, c["precisions"])
            for v in (X, E, M, O):
                v.destroy()
    finally:
        handle.set_policy(None)
        pol.destroy()


def test_crt_toy_key(handle, golden):
    """The sample's CRT decryption sequence (mod, powm, mul, add, mod) recovers the messages."""
    k = golden["crt_toy"]
    cnt = len(k["ciphertexts"])
    C = _arr(handle, 64, k["ciphertexts"])
    P, Q, N = _arr(handle, 32, [k["p"]]), _arr(handle, 32, [k["q"]]), _arr(handle, 64, [k["n"]])
    DP, DQ = _arr(handle, 32, [k["dp"]]), _arr(handle, 32, [k["dq"]])
    CP, CQ = _arr(handle, 64, [k["cp"]]), _arr(handle, 64, [k["cq"]])
    cm, mp, mq = handle.integers(32, cnt), handle.integers(32, cnt), handle.integers(32, cnt)
    sp, sq, r = handle.integers(64, cnt), handle.integers(64, cnt), handle.integers(64, cnt)
    xmp.mod(handle, cm, C, P, cnt)
    xmp.powm(handle, mp, cm, DP, P, cnt)
    xmp.mod(handle, cm, C, Q, cnt)
    xmp.powm(handle, mq, cm, DQ, Q, cnt)
    xmp.mul(handle, sp, mp, CP, cnt)
    xmp.mul(handle, sq, mq, CQ, cnt)
    xmp.add(handle, sp, sp, sq, cnt)
    xmp.mod(handle, r, sp, N, cnt)
    assert ints_from_rows(r.export()) == k["messages"]
    M = _arr(handle, 64, k["messages"])
    assert list(xmp.cmp(handle, M, r, cnt)) == [0] * cnt
