"""Batched mixed-precision powm plans (persistent bins, concurrent streams,
CUDA graph) and CRT items, bit-exact against GMP / Python integers; a plan's
results equal each item computed alone through xmpIntegersPowm."""
import numpy as np
import pytest

import oracle
import xmp_b200 as xmp

pytestmark = pytest.mark.gpu


def _keys(n, half_bits, seed):
    keys = []
    s = seed
    while len(keys) < n:
        p0 = oracle.random_limbs(s, 1, half_bits // 32)[0]
        q0 = oracle.random_limbs(s + 1, 1, half_bits // 32)[0]
        p0[-1] |= np.uint32(0x80000000)
        q0[-1] |= np.uint32(0x80000000)
        s += 2
        k = oracle.crt_key(p0, q0)
        if k is not None and oracle.to_int(k["p"]) != oracle.to_int(k["q"]):
            keys.append(k)
    return keys


def _crt_case(h, nkeys, count, half_bits, seed):
    keys = _keys(nkeys, half_bits, seed)
    hn = half_bits // 32
    rows = {k: np.stack([kk[k] for kk in keys]) for k in ("p", "q", "dp", "dq", "qinv", "n")}
    rng = np.random.default_rng(seed)
    msgs, cts = [], []
    for i in range(count):
        k = keys[i % nkeys]
        n = oracle.to_int(k["n"])
        m = int(rng.integers(0, 2 ** 62)) * (2 ** 60) % n
        msgs.append(m)
        cts.append(pow(m, 65537, n))
    C = h.integers(2 * half_bits, count, np.stack([oracle.from_int(c, 2 * hn) for c in cts]))
    arrs = {k: h.integers(half_bits, nkeys, rows[k]) for k in ("p", "q", "dp", "dq", "qinv")}
    out = h.integers(2 * half_bits, count)
    return msgs, C, arrs, out


@pytest.mark.parametrize("use_graph", [False, True])
def test_mixed_precision_plan_with_crt(handle, use_graph):
    items, expected, arrays = [], [], []
    for bits, count, seed in ((256, 700, 1), (512, 300, 2), (1024, 200, 3), (256, 64, 4)):
        n = bits // 32
        m = oracle.full_length_odd(seed, count, n)
        x = oracle.random_limbs(seed + 10, count, n)
        e = oracle.random_limbs(seed + 20, count, n)
        want, _ = oracle.powm(x, e, m, count)
        X, E, M = [handle.integers(bits, count, v) for v in (x, e, m)]
        O = handle.integers(bits, count)
        items.append((O, X, E, M, count))
        expected.append(want)
        arrays += [X, E, M, O]
    msgs, C, ka, out = _crt_case(handle, 8, 96, 256, 5)
    plan = xmp.BatchPlan(handle, items, [(out, C, ka["p"], ka["q"], ka["dp"], ka["dq"], ka["qinv"], 96)],
                         use_graph=use_graph)
    info = plan.info()
    assert sorted({b["precision"] for b in info}) == [256, 512, 1024]
    for rep in range(2):
        plan.execute()
        for (O, X, E, M, cnt), want in zip(items, expected):
            assert np.array_equal(O.export(), want), (rep, O.precision)
        assert [oracle.to_int(r) for r in out.export()] == msgs, rep
    plan.destroy()
    for a in arrays + [C, out] + list(ka.values()):
        a.destroy()


def test_plan_equals_items_alone(handle):
    """Each item's result in the mixed plan equals the same item run alone."""
    specs = [(2048, 96, 31), (3072, 48, 32), (1024, 200, 33)]
    items, alone, arrays = [], [], []
    for bits, count, seed in specs:
        n = bits // 32
        m = oracle.full_length_odd(seed, count, n)
        x = oracle.below(seed + 1, m)
        e = oracle.random_limbs(seed + 2, count, n)
        X, E, M = [handle.integers(bits, count, v) for v in (x, e, m)]
        O1, O2 = handle.integers(bits, count), handle.integers(bits, count)
        xmp.powm(handle, O1, X, E, M, count)
        alone.append(O1.export())
        items.append((O2, X, E, M, count))
        arrays += [X, E, M, O1, O2]
    plan = xmp.BatchPlan(handle, items, use_graph=True)
    plan.execute()
    for (O2, *_), want in zip(items, alone):
        assert np.array_equal(O2.export(), want)
    plan.destroy()
    for a in arrays:
        a.destroy()


def test_plan_argument_errors(handle):
    """Documented error codes for bad plan arguments; nothing is left allocated."""
    X, E, M = (handle.integers(512, 8, oracle.random_limbs(40 + k, 8, 16)) for k in range(3))
    O_bad = handle.integers(1024, 8)   # precision differs from base/mod
    O_small = handle.integers(512, 4)  # fewer instances than the item's count
    try:
        for items, name in (([(O_bad, X, E, M, 8)], "xmpErrorInvalidPrecision"),
                            ([(O_small, X, E, M, 8)], "xmpErrorInvalidCount")):
            with pytest.raises(xmp.XmpError) as ei:
                xmp.BatchPlan(handle, items)
            assert ei.value.name == name
        # a CRT item whose output is not twice the half size
        p = handle.integers(256, 8, oracle.full_length_odd(50, 8, 8))
        c, out = handle.integers(512, 8), handle.integers(768, 8)
        with pytest.raises(xmp.XmpError) as ei:
            xmp.BatchPlan(handle, [], [(out, c, p, p, p, p, p, 8)])
        assert ei.value.name == "xmpErrorInvalidPrecision"
        for v in (p, c, out):
            v.destroy()
    finally:
        for v in (X, E, M, O_bad, O_small):
            v.destroy()
