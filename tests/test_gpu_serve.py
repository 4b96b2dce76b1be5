"""Continuous-batching modexp server on the GPU.

* Requests of several precisions submitted together (their waves overlap on
  the device) give results bit-identical to GMP, to the same request served
  alone, and to plain xmpIntegersPowm.
* Admission: with op slots for far fewer ops than are queued, every request
  still completes, correctly, and the stalls are counted.
* Open-loop replay through the server and through plain synchronous calls
  give the same results.
* Bad arguments return the documented error codes.
"""
import numpy as np
import pytest

import oracle
import xmp_b200 as xmp

pytestmark = pytest.mark.gpu


def _keys(precision, count, seed):
    return oracle.full_length_odd(seed, count, precision // 32)


def _requests(rng, key_ids, key_rows, n_req, max_ops, seed):
    reqs = []
    for r in range(n_req):
        k = int(rng.integers(0, len(key_ids)))
        m = key_rows[k]
        nops = int(rng.integers(1, max_ops + 1))
        mm = np.repeat(m[None, :], nops, axis=0)
        b = oracle.below(seed + 2 * r, mm)
        e = oracle.random_limbs(seed + 2 * r + 1, nops, m.shape[0])
        reqs.append((key_ids[k], mm, b, e))
    return reqs


def _expected(reqs):
    return [oracle.powm(b, e, mm, mm.shape[0])[0] for _, mm, b, e in reqs]


def test_results_alone_and_in_the_mix(handle):
    rng = np.random.default_rng(5)
    srv = xmp.Server(handle, [1024, 2048, 3072], max_slots=4096, max_keys=64, streams=8)
    try:
        reqs = []
        for prec, seed in ((1024, 100), (2048, 200), (3072, 300)):
            rows = _keys(prec, 6, seed)
            first = srv.add_keys(prec, rows)
            ids = list(range(first, first + len(rows)))
            reqs += _requests(rng, ids, rows, 12, 24, seed + 7)
        order = rng.permutation(len(reqs))
        want = _expected(reqs)
        # all at once: waves of different classes and sizes overlap on the device
        outs = [np.zeros_like(reqs[i][2]) for i in range(len(reqs))]
        rids = {}
        for i in order:
            k, mm, b, e = reqs[i]
            rids[i] = srv.submit(k, b, e, outs[i])
        for i in order:
            assert srv.wait(rids[i], 60_000_000)
        for i in range(len(reqs)):
            assert np.array_equal(outs[i], want[i]), i
        st = srv.stats()
        assert st["requests_completed"] == len(reqs)
        assert st["ops_completed"] == sum(r[2].shape[0] for r in reqs)
        # each alone gives the same result
        for i in range(0, len(reqs), 3):
            k, mm, b, e = reqs[i]
            o = np.zeros_like(b)
            assert srv.wait(srv.submit(k, b, e, o), 60_000_000)
            assert np.array_equal(o, outs[i]), i
        # and plain xmpIntegersPowm agrees
        for i in range(0, len(reqs), 5):
            k, mm, b, e = reqs[i]
            prec = mm.shape[1] * 32
            X, E, M = (handle.integers(prec, len(b), v) for v in (b, e, mm))
            O = handle.integers(prec, len(b))
            xmp.powm(handle, O, X, E, M, len(b))
            assert np.array_equal(O.export(), outs[i]), i
            for v in (X, E, M, O):
                v.destroy()
    finally:
        srv.destroy()


def test_admission_with_few_slots(handle):
    rng = np.random.default_rng(9)
    srv = xmp.Server(handle, [1024], max_slots=128, max_wave_ops=64, max_keys=32, streams=4)
    try:
        rows = _keys(1024, 4, 400)
        first = srv.add_keys(1024, rows)
        reqs = _requests(rng, list(range(first, first + 4)), rows, 24, 64, 500)
        outs = [np.zeros_like(r[2]) for r in reqs]
        rids = [srv.submit(k, b, e, o) for (k, mm, b, e), o in zip(reqs, outs)]
        for rid in rids:
            assert srv.wait(rid, 60_000_000)
        for o, w in zip(outs, _expected(reqs)):
            assert np.array_equal(o, w)
        st = srv.stats()
        assert st["max_inflight_ops"] <= 128
        assert st["admission_stalls"] >= 1
    finally:
        srv.destroy()


def test_replay_server_and_synchronous(handle):
    rng = np.random.default_rng(11)
    srv = xmp.Server(handle, [2048, 1024], max_slots=2048, max_keys=16)
    try:
        r1 = _keys(2048, 3, 600)
        r2 = _keys(1024, 3, 610)
        f1 = srv.add_keys(2048, r1)
        f2 = srv.add_keys(1024, r2)
        reqs = _requests(rng, [f1, f1 + 1, f1 + 2], r1, 10, 8, 700) + \
            _requests(rng, [f2, f2 + 1, f2 + 2], r2, 10, 8, 800)
        reqs = [reqs[i] for i in rng.permutation(len(reqs))]
        arrival = np.cumsum(rng.exponential(200_000.0, size=len(reqs))).astype(np.uint64)
        want = _expected(reqs)
        keys = [r[0] for r in reqs]
        bases = [r[2] for r in reqs]
        exps = [r[3] for r in reqs]
        for mode in (0, 1):
            outs = [np.zeros_like(b) for b in bases]
            lat, secs = srv.replay(keys, arrival, bases, exps, outs, mode=mode)
            assert secs > 0 and np.all(lat > 0)
            for o, w in zip(outs, want):
                assert np.array_equal(o, w), mode
    finally:
        srv.destroy()


def test_errors(handle):
    srv = xmp.Server(handle, [1024], max_slots=256, max_keys=32)
    try:
        even = _keys(1024, 1, 900)
        even[0, 0] &= np.uint32(0xFFFFFFFE)
        for rows, prec, name in ((even, 1024, "xmpErrorInvalidParameter"),
                                 (_keys(2048, 1, 901), 2048, "xmpErrorInvalidPrecision"),
                                 (_keys(1024, 33, 902), 1024, "xmpErrorInvalidCount")):
            with pytest.raises(xmp.XmpError) as ei:
                srv.add_keys(prec, rows)
            assert ei.value.name == name
        first = srv.add_keys(1024, _keys(1024, 2, 903))
        b = np.zeros((1, 32), dtype=np.uint32)
        o = np.zeros_like(b)
        with pytest.raises(xmp.XmpError) as ei:
            srv.submit(first + 2, b, b, o)  # unknown key
        assert ei.value.name == "xmpErrorInvalidParameter"
        rid = xmp.ctypes.c_uint64(0)
        assert xmp.lib().xmpServerSubmit(srv.s, first, 0, b.ctypes.data, b.ctypes.data, o.ctypes.data,
                                         xmp.ctypes.byref(rid)) == 5  # xmpErrorInvalidCount
        with pytest.raises(xmp.XmpError) as ei:
            srv.wait(123456789)
        assert ei.value.name == "xmpErrorInvalidParameter"
    finally:
        srv.destroy()


def test_concurrent_submitters(handle):
    """Submit and Wait from several host threads at once (ctypes releases the GIL in the calls)."""
    import threading
    srv = xmp.Server(handle, [1024, 2048], max_slots=2048, max_keys=16, streams=8)
    try:
        r1, r2 = _keys(1024, 4, 1000), _keys(2048, 4, 1010)
        f1, f2 = srv.add_keys(1024, r1), srv.add_keys(2048, r2)
        per_thread = []
        for t in range(4):
            rng = np.random.default_rng(1100 + t)
            per_thread.append(_requests(rng, [f1, f1 + 1, f1 + 2, f1 + 3], r1, 6, 12, 1200 + 100 * t) +
                              _requests(rng, [f2, f2 + 1, f2 + 2, f2 + 3], r2, 4, 12, 1250 + 100 * t))
        results, errors = {}, []

        def worker(t):
            try:
                outs = []
                for k, mm, b, e in per_thread[t]:
                    o = np.zeros_like(b)
                    outs.append((srv.submit(k, b, e, o), o))
                for rid, o in outs:
                    assert srv.wait(rid, 60_000_000)
                results[t] = [o for _, o in outs]
            except Exception as ex:  # reported on the main thread
                errors.append(ex)

        threads = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
        for th in threads:
            th.start()
        for th in threads:
            th.join(120)
        assert not errors, errors
        for t in range(4):
            for got, want in zip(results[t], _expected(per_thread[t])):
                assert np.array_equal(got, want)
        assert srv.stats()["requests_completed"] == sum(len(p) for p in per_thread)
    finally:
        srv.destroy()


def test_wait_timeout_and_poll(handle):
    """Wait with a short timeout (or 0: a poll) reports not-done without retiring the request;
    a later wait collects the result."""
    srv = xmp.Server(handle, [4096], max_slots=256, max_keys=32, streams=2)
    try:
        m = _keys(4096, 1, 1300)
        k = srv.add_keys(4096, m)
        mm = np.repeat(m, 2, axis=0)
        b = oracle.below(1301, mm)
        e = oracle.random_limbs(1302, 2, 128)
        out = np.zeros_like(b)
        rid = srv.submit(k, b, e, out)
        assert not srv.wait(rid, 0)        # a 4096-bit exponentiation takes tens of milliseconds
        assert not srv.wait(rid, 100)      # 0.1 ms is not enough either
        assert srv.wait(rid, 60_000_000)
        assert np.array_equal(out, oracle.powm(b, e, mm, 2)[0])
        with pytest.raises(xmp.XmpError):
            srv.wait(rid, 0)               # retired once reported done
    finally:
        srv.destroy()
