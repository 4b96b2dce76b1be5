"""Autotuner and learned selector on the GPU.

* The CUDA backward pass matches the float64 numpy restatement
  (oracle/selector_ref.py, itself pinned to finite differences on the CPU).
* CUDA training lowers the loss; CUDA prediction matches the restatement.
* A loaded selector's grid table (one network, or an ensemble's mean
  prediction) drives xmpIntegersPowm choices, and results
  stay bit-exact whatever configuration is chosen.
* With the committed dataset (exhaustive-tuner timings on a B200) and weights,
  the selector's regret on the held-out shapes is lower than the built-in
  heuristic's and within 5%.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle
import xmp_b200 as xmp
from oracle import selector_ref as ref
from xmp_b200 import tuning

pytestmark = pytest.mark.gpu


def _data(seed, n=40):
    rng = np.random.default_rng(seed)
    shapes = [(int(rng.integers(0, 3)), int(32 * rng.integers(4, 128)), int(rng.integers(0, 4096)),
               int(2 ** rng.integers(6, 20))) for _ in range(n)]
    ms = rng.uniform(0.01, 50.0, size=(n, 48)).astype(np.float32)
    ms[rng.uniform(size=ms.shape) < 0.3] = -1.0
    return shapes, ms


def test_cuda_gradients_match_restatement(handle):
    shapes, ms = _data(1)
    p = ref.init(2).astype(np.float32)
    loss, g = tuning.gradients(handle, p, shapes, ms)
    rloss, rg = ref.loss_and_grad(p.astype(np.float64), shapes, ms)
    assert abs(loss - rloss) <= 1e-4 * max(1.0, abs(rloss))
    assert np.allclose(g, rg, rtol=2e-3, atol=2e-4 * np.abs(rg).max())


def test_cuda_training_and_prediction(handle):
    shapes, ms = _data(3, n=64)
    p0 = ref.init(5).astype(np.float32)
    l0, _ = ref.loss_and_grad(p0, shapes, ms)
    p, loss = tuning.train(handle, shapes, ms, epochs=300, lr=3e-3, seed=0, params=p0)
    assert loss < 0.5 * l0
    pred = tuning.predict(handle, p, shapes)
    _, _, want = ref.forward(p.astype(np.float64), ref.features(shapes))
    assert np.allclose(pred, want, rtol=1e-4, atol=1e-3)


def test_exhaustive_tuner_and_choice_drive_powm(handle):
    shape = (tuning.OPS["powm"], 512, 128, 512)
    ms = tuning.measure(handle, shape, reps=1)
    valid = tuning.candidate_valid(shape[0], shape[1])
    for s in range(48):
        if valid[s]:
            assert np.isnan(ms[s]) or ms[s] > 0
        else:
            assert ms[s] < 0
    best = int(np.nanargmin(np.where(ms > 0, ms, np.nan)))
    sh = tuning.Shape(*shape)
    xmp.check(xmp.lib().xmpTuneSetChoice(handle.h, ctypes.byref(sh), best))
    slot, src = ctypes.c_int32(), ctypes.c_int32()
    xmp.check(xmp.lib().xmpTuneGetChoice(handle.h, ctypes.byref(sh), ctypes.byref(slot), ctypes.byref(src)))
    assert (slot.value, src.value) == (best, 1)
    # results through the tuned choice and through every valid candidate are bit-exact
    m = oracle.full_length_odd(9, 512, 16)
    x = oracle.below(10, m)
    e = oracle.random_limbs(11, 512, 4)
    want, _ = oracle.powm(x, e, m, 512)
    X, E, M, O = handle.integers(512, 512, x), handle.integers(128, 512, e), handle.integers(512, 512, m), \
        handle.integers(512, 512)
    xmp.powm(handle, O, X, E, M, 512)
    assert np.array_equal(O.export(), want)
    for s in range(0, 42, 5):
        cfg = xmp.PowmConfig()
        v = ctypes.c_int32()
        xmp.check(xmp.lib().xmpTuneCandidate(shape[0], 512, s, ctypes.byref(v), ctypes.byref(cfg)))
        if v.value:
            xmp.powm_with_config(handle, O, X, E, M, 512, cfg)
            assert np.array_equal(O.export(), want), cfg
    xmp.check(xmp.lib().xmpTuneClear(handle.h))
    for v_ in (X, E, M, O):
        v_.destroy()


@pytest.mark.parametrize("members", [1, 3])
def test_selector_table_lookup(handle, members):
    shapes, ms = _data(7, n=64)
    p, _ = tuning.train_ensemble(handle, shapes, ms, members=members, epochs=100, lr=3e-3, seed=1)
    tuning.install(handle, p)
    try:
        probe = [(2, 2048, 2048, 65536), (2, 1024, 17, 4096), (0, 512, 0, 1 << 18), (1, 1024, 0, 1 << 18)]
        for sh in probe:
            slot, src = ctypes.c_int32(), ctypes.c_int32()
            xmp.check(xmp.lib().xmpTuneGetChoice(handle.h, ctypes.byref(tuning.Shape(*sh)), ctypes.byref(slot),
                                                 ctypes.byref(src)))
            assert src.value == 2
            valid = tuning.candidate_valid(sh[0], sh[1])
            assert valid[slot.value]
            # the grid cell's representative point (geometric middle of its count / exponent
            # buckets) predicts this slot as the best valid one
            cb = max(int(np.floor(np.log2(sh[3]))), 6)  # batches below 2^6 take the 2^6 cell
            eb = int(np.floor(np.log2(max(sh[2], 1))))
            x = np.array([[sh[0] - 1.0, (np.log2(sh[1]) - 10.0) / 4.0, (cb + 0.5 - 13.0) / 7.0,
                           (eb + 0.5 - 7.0) / 7.0 if sh[0] == 2 else -1.0]])
            # an ensemble's table follows the members' mean prediction
            pred = np.mean([ref.forward(m.astype(np.float64), x)[2][0] for m in tuning.members_of(p)], axis=0)
            masked = np.where(valid, pred, np.inf)
            assert pred[slot.value] <= masked.min() + 1e-3
    finally:
        xmp.check(xmp.lib().xmpTuneClear(handle.h))


@pytest.mark.skipif(not (os.path.exists(tuning.DEFAULT_DATA) and os.path.exists(tuning.DEFAULT_WEIGHTS)),
                    reason="no committed tuning dataset / selector weights")
def test_committed_selector_beats_heuristic(handle):
    """The compiled-in selector was trained on 80% of the measured shapes; on the other 20% (batch
    sizes and exponent lengths it has not seen, at the measured precisions) its choices cost less
    than the built-in heuristic's, and stay within the 5% regret target."""
    shapes, ms, _ = tuning.load_dataset(tuning.DEFAULT_DATA)
    params = tuning.load_weights()
    tr, te = tuning.splits(shapes)["shapes"]
    r = tuning.evaluate(handle, params, shapes, ms, te)
    assert r["selector_mean_regret"] <= r["heuristic_mean_regret"] + 1e-9, r
    assert r["selector_mean_regret"] <= 0.05, r
